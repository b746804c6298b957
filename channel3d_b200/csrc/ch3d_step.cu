// ch3d_step.cu -- sm_100a kernels of the 2nd-order partially implicit RK3
// step (src/CFD_2nd/m_ChannelSystem.f90:73-154 with the PIMP procedures of
// src/CFD_2nd/m_TSchemePIMP_inc.f90) and the pressure Poisson pipeline
// (src/CFD_2nd/m_Poisson.f90:1078-1201).  FP64 and FP32 (mixed) instances.
//
// Per substep the device runs:
//   substep_setup  PMcoeUpdate + bulk-velocity reduction (clcRhsX_PIMP :60-74)
//   rhs + uhat     clcRhsX/Y/Z_PIMP and clcU1/2/3Hat_PIMP as one column march
//                  (ch3d_march.cu); the stage entry points run them separately
//                  (k_rhs_pimp, k_uhat_pimp: partitioned tridiagonal)
//   prsrc_xfft     clcPrSrcOther fused with the forward x R2C FFT
//   spectral       z FFT, y tridiagonal per (kx,kz) with the (0,0) pin, z iFFT
//   xifft          x C2R FFT * normfft -> phi
//   proj           FluidVelUpdate + PressureUpdate_PIMP + next bulk partial sums
// and per step: step_begin (CalcMaxCFL/dt), diag (CheckDivergence, CalcVmax,
// CalcUxAver, next CFL), step_end (limit checks).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

// ---------------------------------------------------------------------------
// scalar kernels
// ---------------------------------------------------------------------------

// src/CFD_2nd/m_ChannelSystem.f90:81-88 (CalcMaxCFL result -> cflmp, dt)
__global__ void k_step_begin(DevScalars* sc, int iCFL, double CFLc, double dtMax) {
  if (sc->status) return;
  double uddx = __longlong_as_double((long long)sc->uddx);
  sc->itime += 1;
  sc->cflmp = uddx * sc->dt;
  if (iCFL == 1) {
    double d = CFLc / uddx;
    sc->dt = d < dtMax ? d : dtMax;
  } else {
    sc->dt = dtMax;
  }
}

// src/CFD_2nd/m_Parameters.f90:329-342 (PMcoeUpdate) and the bulk constraint of
// src/CFD_2nd/m_TSchemePIMP_inc.f90:60-74 from the partial sums of the current ux.
// 4th order (order == 4): the partial sums are those of the mean viscous stress
// and the forcing follows src/CFD_4th/m_TScheme.f90:364-377.
__global__ void k_substep_setup(DevScalars* sc, const double* __restrict__ part, int npart, int ns, double gam,
                                double the, double alp, double xnu, int IsUxConst, double ubulk, double norm_bulk,
                                int order, double nxnz, double yly) {
  __shared__ double red[256];
  if (sc->status) return;
  double s = 0;
  for (int q = threadIdx.x; q < npart; q += blockDim.x) s += part[q];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double dt = sc->dt;
    sc->pmGamma = gam * dt;
    sc->pmTheta = the * dt;
    sc->pmAlpha = alp * dt;
    sc->pmBeta = 0.5 * alp * xnu * dt;
    sc->SimTime = sc->SimTime + dt * alp;
    sc->pmAlphaC = alp;
    sc->pmBetaT = 0.5 * alp * dt;
    if (ns == 1) sc->PrGradAver = 0.0;
    sc->ns = ns;
    sc->divmax1 = 0ull;
    if (IsUxConst && order == 4) {
      const double dpm = xnu * red[0] / nxnz / yly;
      sc->PrGradNow = dpm;
      sc->dpmdxns = -(sc->pmAlpha * dpm);  // RhsX - pmAlpha*dpmdxns
      sc->PrGradAver = sc->PrGradAver + dpm * alp;
    } else if (IsUxConst) {
      double s1tot1 = red[0] * norm_bulk;
      sc->s1tot1 = s1tot1;
      sc->dpmdxns = alp * (ubulk - s1tot1);
      sc->PrGradNow = (ubulk - s1tot1) / dt;
      sc->PrGradAver = sc->PrGradAver + alp * sc->PrGradNow;
    } else {
      sc->dpmdxns = 0.0;
    }
  }
}

// src/CFD_2nd/m_ChannelSystem.f90:127-130 (limit checks after the step) and
// CalcUxAver (src/CFD_2nd/m_Tools.f90:250-270) from partial sums.
__global__ void k_step_end(DevScalars* sc, const double* __restrict__ part, int npart, double norm_uxm, double div_limit,
                           double vel_limit) {
  __shared__ double red[256];
  if (sc->status) return;
  double s = 0;
  for (int q = threadIdx.x; q < npart; q += blockDim.x) s += part[q];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sc->uxm = red[0] * norm_uxm;
    double d2 = __longlong_as_double((long long)sc->divmax2);
    double v0 = __longlong_as_double((long long)sc->vmax[0]);
    double v1 = __longlong_as_double((long long)sc->vmax[1]);
    double v2 = __longlong_as_double((long long)sc->vmax[2]);
    double vmin = fmin(v0, fmin(v1, v2));
    if (!(d2 <= div_limit)) sc->status = 1;        // NaN trips too
    else if (!(vmin <= vel_limit)) sc->status = 2;
  }
}

// ---------------------------------------------------------------------------
// clcRhsX/Y/Z_PIMP  (src/CFD_2nd/m_TSchemePIMP_inc.f90:7-75, 161-209, 277-325)
// at one cell: returns the three right-hand sides and updates HistX/Y/Z.
// The mean pressure gradient dpmdxns (:61-74) is added by the callers.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void rhs_point(const Geo<T>& g, const Metrics<T>& m, const T* __restrict__ ux,
                                          const T* __restrict__ uy, const T* __restrict__ uz,
                                          const T* __restrict__ pr, T* __restrict__ hx, T* __restrict__ hy,
                                          T* __restrict__ hz, int i, int j, int k, T pmGamma, T pmTheta, T pmAlpha,
                                          T pmBeta, T& rxo, T& ryo, T& rzo) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int im = wrapm(i, nx), ip = wrapp(i, nx), km = wrapm(k, nz), kp = wrapp(k, nz);
  const int jc = j + 1;
  const T two = (T)2, half = (T)0.5, quarter = (T)0.25, one = (T)1;
  const long long idx = i + (long long)nx * (j + (long long)ny * k);

  const T ux_c = __ldg(ux + idx);
  const T ux_ip = fld(ux, g, 0, ip, j, k), ux_im = fld(ux, g, 0, im, j, k);
  const T ux_jp = fld(ux, g, 0, i, j + 1, k), ux_jm = fld(ux, g, 0, i, j - 1, k);
  const T ux_kp = fld(ux, g, 0, i, j, kp), ux_km = fld(ux, g, 0, i, j, km);
  const T ux_ip_jm = fld(ux, g, 0, ip, j - 1, k), ux_ip_km = fld(ux, g, 0, ip, j, km);
  const T uy_c = __ldg(uy + idx);
  const T uy_ip = fld(uy, g, 1, ip, j, k), uy_im = fld(uy, g, 1, im, j, k);
  const T uy_jp = fld(uy, g, 1, i, j + 1, k), uy_jm = fld(uy, g, 1, i, j - 1, k);
  const T uy_im_jp = fld(uy, g, 1, im, j + 1, k);
  const T uy_kp = fld(uy, g, 1, i, j, kp), uy_km = fld(uy, g, 1, i, j, km);
  const T uy_jp_km = fld(uy, g, 1, i, j + 1, km);
  const T uz_c = __ldg(uz + idx);
  const T uz_ip = fld(uz, g, 2, ip, j, k), uz_im = fld(uz, g, 2, im, j, k);
  const T uz_jp = fld(uz, g, 2, i, j + 1, k), uz_jm = fld(uz, g, 2, i, j - 1, k);
  const T uz_kp = fld(uz, g, 2, i, j, kp), uz_km = fld(uz, g, 2, i, j, km);
  const T uz_im_kp = fld(uz, g, 2, im, j, kp), uz_jm_kp = fld(uz, g, 2, i, j - 1, kp);
  const T p_c = __ldg(pr + idx);
  const T p_im = fld(pr, g, 3, im, j, k), p_jm = fld(pr, g, 3, i, j - 1, k), p_km = fld(pr, g, 3, i, j, km);
  const T hx_o = hx[idx], hy_o = hy[idx], hz_o = hz[idx];

  const T rdx = g.rdx, rdz = g.rdz, rdx2 = g.rdx2, rdz2 = g.rdz2, xnu = g.xnu;
  const T IY1 = m.yinterp[jc], IY2 = one - IY1;
  const T IY3 = m.yinterp[jc + 1], IY4 = one - IY3;
  {  // RhsX
    const T qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    const T sucaj = half * m.rdyp[jc];
    T h11 = ((ux_ip + ux_c) * (ux_ip + ux_c) - (ux_c + ux_im) * (ux_c + ux_im)) * qdx1;
    T h12 = ((uy_jp + uy_im_jp) * (IY3 * ux_c + IY4 * ux_jp) - (uy_c + uy_im) * (IY1 * ux_jm + IY2 * ux_c)) * sucaj;
    T h13 = ((uz_kp + uz_im_kp) * (ux_kp + ux_c) - (uz_c + uz_im) * (ux_c + ux_km)) * qdx3;
    T d11q1 = (ux_ip - two * ux_c + ux_im) * rdx2;
    T d22q1 = m.ap2c[jc] * ux_jp + m.ac2c[jc] * ux_c + m.am2c[jc] * ux_jm;
    T d33q1 = g.ap3c * ux_kp + g.ac3c * ux_c + g.am3c * ux_km;
    T dcq13 = d11q1 + d33q1;
    T gradp1 = (p_c - p_im) * rdx;
    T convEd1 = -h11 - h12 - h13 + xnu * dcq13 + g.g1;
    rxo = pmGamma * convEd1 + pmTheta * hx_o - pmAlpha * gradp1 + two * pmBeta * d22q1;
    hx[idx] = convEd1;
  }
  {  // RhsY
    const T hdx1 = half * rdx, hdx3 = half * rdz;
    const T sucac = m.rdyc[jc], qsucac = quarter * sucac;
    T h21 = ((IY1 * ux_ip_jm + IY2 * ux_ip) * (uy_ip + uy_c) - (IY1 * ux_jm + IY2 * ux_c) * (uy_c + uy_im)) * hdx1;
    T h22 = ((uy_jp + uy_c) * (uy_jp + uy_c) - (uy_c + uy_jm) * (uy_c + uy_jm)) * qsucac;
    T h23 = ((IY1 * uz_jm_kp + IY2 * uz_kp) * (uy_kp + uy_c) - (IY1 * uz_jm + IY2 * uz_c) * (uy_c + uy_km)) * hdx3;
    T d11q2 = g.ap1c * uy_ip + g.ac1c * uy_c + g.am1c * uy_im;
    T d22q2 = m.ap2p[jc] * uy_jp + m.ac2p[jc] * uy_c + m.am2p[jc] * uy_jm;
    T d33q2 = g.ap3c * uy_kp + g.ac3c * uy_c + g.am3c * uy_km;
    T dcq13 = d11q2 + d33q2;
    T gradp2 = (p_c - p_jm) * sucac;
    T convEd2 = -h21 - h22 - h23 + xnu * dcq13 + g.g2;
    ryo = pmGamma * convEd2 + pmTheta * hy_o - pmAlpha * gradp2 + two * pmBeta * d22q2;
    hy[idx] = convEd2;
  }
  {  // RhsZ
    const T qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    const T sucaj = half * m.rdyp[jc];
    T h31 = ((ux_ip + ux_ip_km) * (uz_ip + uz_c) - (ux_c + ux_km) * (uz_c + uz_im)) * qdx1;
    T h32 = ((uy_jp + uy_jp_km) * (IY3 * uz_c + IY4 * uz_jp) - (uy_c + uy_km) * (IY1 * uz_jm + IY2 * uz_c)) * sucaj;
    T h33 = ((uz_kp + uz_c) * (uz_kp + uz_c) - (uz_c + uz_km) * (uz_c + uz_km)) * qdx3;
    T d11q3 = g.ap1c * uz_ip + g.ac1c * uz_c + g.am1c * uz_im;
    T d22q3 = m.ap2c[jc] * uz_jp + m.ac2c[jc] * uz_c + m.am2c[jc] * uz_jm;
    T d33q3 = (uz_kp - two * uz_c + uz_km) * rdz2;
    T dcq13 = d11q3 + d33q3;
    T gradp3 = (p_c - p_km) * rdz;
    T convEd3 = -h31 - h32 - h33 + xnu * dcq13 + g.g3;
    rzo = pmGamma * convEd3 + pmTheta * hz_o - pmAlpha * gradp3 + two * pmBeta * d22q3;
    hz[idx] = convEd3;
  }
}

// One component of clcRhsX/Y/Z_PIMP (or _FIMP, _FEXP) at one cell (C = 0, 1, 2),
// with its Hist update.
template <class T, int C>
__device__ __forceinline__ T rhs_comp(const Geo<T>& g, const Metrics<T>& m, const T* __restrict__ ux,
                                      const T* __restrict__ uy, const T* __restrict__ uz, const T* __restrict__ pr,
                                      T* __restrict__ h, int i, int j, int k, T pmGamma, T pmTheta, T pmAlpha,
                                      T pmBeta) {
  const Nbr n = make_nbr(g, i, j, k);
  const int jc = j + 1;
  const T two = (T)2, half = (T)0.5, quarter = (T)0.25, one = (T)1;
  const T rdx = g.rdx, rdz = g.rdz, rdx2 = g.rdx2, rdz2 = g.rdz2, xnu = g.xnu;
  const T IY1 = m.yinterp[jc], IY2 = one - IY1;
  if (C == 0) {
    const T ux_c = at(ux, n, 0), ux_ip = at(ux, n, n.xp), ux_im = at(ux, n, n.xm);
    const T ux_jp = at_jp(ux, g, 0, n, 0), ux_jm = at_jm(ux, g, 0, n, 0);
    const T ux_kp = at(ux, n, n.zp), ux_km = at(ux, n, n.zm);
    const T uy_c = at(uy, n, 0), uy_im = at(uy, n, n.xm);
    const T uy_jp = at_jp(uy, g, 1, n, 0), uy_im_jp = at_jp(uy, g, 1, n, n.xm);
    const T uz_c = at(uz, n, 0), uz_im = at(uz, n, n.xm);
    const T uz_kp = at(uz, n, n.zp), uz_im_kp = at(uz, n, n.zp + n.xm);
    const T p_c = at(pr, n, 0), p_im = at(pr, n, n.xm);
    const T h_o = h[n.c];
    const T IY3 = m.yinterp[jc + 1], IY4 = one - IY3;
    const T qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    const T sucaj = half * m.rdyp[jc];
    T h11 = ((ux_ip + ux_c) * (ux_ip + ux_c) - (ux_c + ux_im) * (ux_c + ux_im)) * qdx1;
    T h12 = ((uy_jp + uy_im_jp) * (IY3 * ux_c + IY4 * ux_jp) - (uy_c + uy_im) * (IY1 * ux_jm + IY2 * ux_c)) * sucaj;
    T h13 = ((uz_kp + uz_im_kp) * (ux_kp + ux_c) - (uz_c + uz_im) * (ux_c + ux_km)) * qdx3;
    T d11q1 = (ux_ip - two * ux_c + ux_im) * rdx2;
    T d22q1 = m.ap2c[jc] * ux_jp + m.ac2c[jc] * ux_c + m.am2c[jc] * ux_jm;
    T d33q1 = g.ap3c * ux_kp + g.ac3c * ux_c + g.am3c * ux_km;
    T dcq13 = d11q1 + d33q1;
    T gradp1 = (p_c - p_im) * rdx;
    if (g.implicit == 0) {  // clcRhsX_FEXP (src/CFD_2nd/m_TSchemeFEXP_inc.f90:33-55)
      T convEd1 = -h11 - h12 - h13 + xnu * (d11q1 + d22q1 + d33q1) + g.g1;
      h[n.c] = convEd1;
      return pmGamma * convEd1 + pmTheta * h_o - pmAlpha * gradp1;
    }
    if (g.implicit == 2) {  // clcRhsX_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:45-55)
      T convEd1 = -h11 - h12 - h13 + g.g1;
      h[n.c] = convEd1;
      return pmGamma * convEd1 + pmTheta * h_o - pmAlpha * gradp1 + two * pmBeta * (d11q1 + d22q1 + d33q1);
    }
    T convEd1 = -h11 - h12 - h13 + xnu * dcq13 + g.g1;
    h[n.c] = convEd1;
    return pmGamma * convEd1 + pmTheta * h_o - pmAlpha * gradp1 + two * pmBeta * d22q1;
  } else if (C == 1) {
    const T ux_c = at(ux, n, 0), ux_ip = at(ux, n, n.xp);
    const T ux_jm = at_jm(ux, g, 0, n, 0), ux_ip_jm = at_jm(ux, g, 0, n, n.xp);
    const T uy_c = at(uy, n, 0), uy_ip = at(uy, n, n.xp), uy_im = at(uy, n, n.xm);
    const T uy_jp = at_jp(uy, g, 1, n, 0), uy_jm = at_jm(uy, g, 1, n, 0);
    const T uy_kp = at(uy, n, n.zp), uy_km = at(uy, n, n.zm);
    const T uz_c = at(uz, n, 0), uz_jm = at_jm(uz, g, 2, n, 0);
    const T uz_kp = at(uz, n, n.zp), uz_jm_kp = at_jm(uz, g, 2, n, n.zp);
    const T p_c = at(pr, n, 0), p_jm = at_jm(pr, g, 3, n, 0);
    const T h_o = h[n.c];
    const T hdx1 = half * rdx, hdx3 = half * rdz;
    const T sucac = m.rdyc[jc], qsucac = quarter * sucac;
    T h21 = ((IY1 * ux_ip_jm + IY2 * ux_ip) * (uy_ip + uy_c) - (IY1 * ux_jm + IY2 * ux_c) * (uy_c + uy_im)) * hdx1;
    T h22 = ((uy_jp + uy_c) * (uy_jp + uy_c) - (uy_c + uy_jm) * (uy_c + uy_jm)) * qsucac;
    T h23 = ((IY1 * uz_jm_kp + IY2 * uz_kp) * (uy_kp + uy_c) - (IY1 * uz_jm + IY2 * uz_c) * (uy_c + uy_km)) * hdx3;
    T d11q2 = g.ap1c * uy_ip + g.ac1c * uy_c + g.am1c * uy_im;
    T d22q2 = m.ap2p[jc] * uy_jp + m.ac2p[jc] * uy_c + m.am2p[jc] * uy_jm;
    T d33q2 = g.ap3c * uy_kp + g.ac3c * uy_c + g.am3c * uy_km;
    T dcq13 = d11q2 + d33q2;
    T gradp2 = (p_c - p_jm) * sucac;
    if (g.implicit == 0) {  // clcRhsY_FEXP (src/CFD_2nd/m_TSchemeFEXP_inc.f90:183-204)
      T convEd2 = -h21 - h22 - h23 + xnu * (d11q2 + d22q2 + d33q2) + g.g2;
      h[n.c] = convEd2;
      return pmGamma * convEd2 + pmTheta * h_o - pmAlpha * gradp2;
    }
    if (g.implicit == 2) {  // clcRhsY_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:104-115)
      T convEd2 = -h21 - h22 - h23 + g.g2;
      h[n.c] = convEd2;
      return pmGamma * convEd2 + pmTheta * h_o - pmAlpha * gradp2 + two * pmBeta * (d11q2 + d22q2 + d33q2);
    }
    T convEd2 = -h21 - h22 - h23 + xnu * dcq13 + g.g2;
    h[n.c] = convEd2;
    return pmGamma * convEd2 + pmTheta * h_o - pmAlpha * gradp2 + two * pmBeta * d22q2;
  } else {
    const T ux_c = at(ux, n, 0), ux_ip = at(ux, n, n.xp);
    const T ux_km = at(ux, n, n.zm), ux_ip_km = at(ux, n, n.zm + n.xp);
    const T uy_c = at(uy, n, 0), uy_jp = at_jp(uy, g, 1, n, 0);
    const T uy_km = at(uy, n, n.zm), uy_jp_km = at_jp(uy, g, 1, n, n.zm);
    const T uz_c = at(uz, n, 0), uz_ip = at(uz, n, n.xp), uz_im = at(uz, n, n.xm);
    const T uz_jp = at_jp(uz, g, 2, n, 0), uz_jm = at_jm(uz, g, 2, n, 0);
    const T uz_kp = at(uz, n, n.zp), uz_km = at(uz, n, n.zm);
    const T p_c = at(pr, n, 0), p_km = at(pr, n, n.zm);
    const T h_o = h[n.c];
    const T IY3 = m.yinterp[jc + 1], IY4 = one - IY3;
    const T qdx1 = quarter * rdx, qdx3 = quarter * rdz;
    const T sucaj = half * m.rdyp[jc];
    T h31 = ((ux_ip + ux_ip_km) * (uz_ip + uz_c) - (ux_c + ux_km) * (uz_c + uz_im)) * qdx1;
    T h32 = ((uy_jp + uy_jp_km) * (IY3 * uz_c + IY4 * uz_jp) - (uy_c + uy_km) * (IY1 * uz_jm + IY2 * uz_c)) * sucaj;
    T h33 = ((uz_kp + uz_c) * (uz_kp + uz_c) - (uz_c + uz_km) * (uz_c + uz_km)) * qdx3;
    T d11q3 = g.ap1c * uz_ip + g.ac1c * uz_c + g.am1c * uz_im;
    T d22q3 = m.ap2c[jc] * uz_jp + m.ac2c[jc] * uz_c + m.am2c[jc] * uz_jm;
    T d33q3 = (uz_kp - two * uz_c + uz_km) * rdz2;
    T dcq13 = d11q3 + d33q3;
    T gradp3 = (p_c - p_km) * rdz;
    if (g.implicit == 0) {  // clcRhsZ_FEXP (src/CFD_2nd/m_TSchemeFEXP_inc.f90:299-320)
      T convEd3 = -h31 - h32 - h33 + xnu * (d11q3 + d22q3 + d33q3) + g.g3;
      h[n.c] = convEd3;
      return pmGamma * convEd3 + pmTheta * h_o - pmAlpha * gradp3;
    }
    if (g.implicit == 2) {  // clcRhsZ_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:161-172)
      T convEd3 = -h31 - h32 - h33 + g.g3;
      h[n.c] = convEd3;
      return pmGamma * convEd3 + pmTheta * h_o - pmAlpha * gradp3 + two * pmBeta * (d11q3 + d22q3 + d33q3);
    }
    T convEd3 = -h31 - h32 - h33 + xnu * dcq13 + g.g3;
    h[n.c] = convEd3;
    return pmGamma * convEd3 + pmTheta * h_o - pmAlpha * gradp3 + two * pmBeta * d22q3;
  }
}

// Stand-alone clcRhsX/Y/Z (one thread per cell); the stage-level entry point.
template <class T>
__global__ void __launch_bounds__(256) k_rhs_pimp(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                  const T* __restrict__ uy, const T* __restrict__ uz,
                                                  const T* __restrict__ pr, T* __restrict__ hx, T* __restrict__ hy,
                                                  T* __restrict__ hz, T* __restrict__ rx, T* __restrict__ ry,
                                                  T* __restrict__ rz, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  T a, b, c;
  rhs_point(g, m, ux, uy, uz, pr, hx, hy, hz, i, j, k, (T)sc->pmGamma, (T)sc->pmTheta, (T)sc->pmAlpha,
            (T)sc->pmBeta, a, b, c);
  const long long idx = i + (long long)g.nx * (j + (long long)g.ny * k);
  rx[idx] = a; ry[idx] = b; rz[idx] = c;
}

// clcRhsX/Y/Z_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:6-177), or _FEXP
// (src/CFD_2nd/m_TSchemeFEXP_inc.f90:6-324) when g.implicit = 0, one thread per
// cell and component (blockIdx.z = component * nz + k: a thread holds one
// component's stencil, so more threads fit an SM than with all three),
// RhsX with the mean pressure gradient (:57-66) included.
template <class T>
__global__ void __launch_bounds__(256) k_rhs_fimp(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                  const T* __restrict__ uy, const T* __restrict__ uz,
                                                  const T* __restrict__ pr, T* __restrict__ hx, T* __restrict__ hy,
                                                  T* __restrict__ hz, T* __restrict__ rx, T* __restrict__ ry,
                                                  T* __restrict__ rz, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int comp = blockIdx.z / g.nz, k = blockIdx.z - comp * g.nz;
  if (i >= g.nx || j >= g.ny) return;
  const T pmGamma = (T)sc->pmGamma, pmTheta = (T)sc->pmTheta, pmAlpha = (T)sc->pmAlpha, pmBeta = (T)sc->pmBeta;
  const long long idx = i + (long long)g.nx * (j + (long long)g.ny * k);
  if (comp == 0)
    rx[idx] = rhs_comp<T, 0>(g, m, ux, uy, uz, pr, hx, i, j, k, pmGamma, pmTheta, pmAlpha, pmBeta) + (T)sc->dpmdxns;
  else if (comp == 1)
    ry[idx] = rhs_comp<T, 1>(g, m, ux, uy, uz, pr, hy, i, j, k, pmGamma, pmTheta, pmAlpha, pmBeta);
  else
    rz[idx] = rhs_comp<T, 2>(g, m, ux, uy, uz, pr, hz, i, j, k, pmGamma, pmTheta, pmAlpha, pmBeta);
}

// Precomputes the chunk factors, spikes and interface block-Thomas factors of
// both Helmholtz sets for the current pmBeta (once per substep; block = set).
__global__ void k_helm_factors(HelmCoef hc, int ny, int P, double* __restrict__ fac,
                               const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int set = blockIdx.x;
  double* F = fac + (size_t)set * helm_set_stride(ny, P);
  double *RM = F, *AA = F + ny, *CP = F + 2 * ny, *AL = F + 3 * ny, *BE = F + 4 * ny, *IFD = F + 5 * ny;
  const double pmBeta = sc->pmBeta;
  const int Q = P - 1;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    const int s = chunk_lo(p, ny, P), e = chunk_hi(p, ny, P);
    double cpp = 0.0, dal = 0.0;
    for (int j = s; j <= e; ++j) {
      double a, b, c;
      helm_abc(hc, set, pmBeta, j, a, b, c);
      const double mm = (j == s) ? b : b - a * cpp;
      const double rm = 1.0 / mm;
      const double cp = c * rm;
      dal = (j == s) ? -a * rm : -a * dal * rm;
      RM[j] = rm; CP[j] = cp; AL[j] = (p == 0) ? 0.0 : dal; AA[j] = a;
      cpp = cp;
    }
    BE[e] = (p == P - 1) ? 0.0 : -CP[e];
    for (int j = e - 1; j >= s; --j) {
      AL[j] = AL[j] - CP[j] * AL[j + 1];
      BE[j] = -CP[j] * BE[j + 1];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m01p = 0.0, vprev = 0.0;
    for (int q = 0; q < Q; ++q) {
      const int eq = chunk_hi(q, ny, P), sq1 = chunk_lo(q + 1, ny, P);
      const double l = -AL[eq], v = -BE[sq1];
      double d00 = 1.0, d01 = -BE[eq], d10 = -AL[sq1], d11 = 1.0;
      if (q > 0) d01 -= l * m01p * vprev;  // (L_q Minv_{q-1} U_{q-1}) has only a (0,1) entry
      const double r = 1.0 / (d00 * d11 - d01 * d10);
      double* R = IFD + 6 * q;
      R[0] = d11 * r; R[1] = -d01 * r; R[2] = -d10 * r; R[3] = d00 * r; R[4] = l; R[5] = v;
      m01p = R[1]; vprev = v;
    }
  }
}

// clcU1Hat/U2Hat/U3Hat_PIMP from RhsX/Y/Z in memory (stage-level entry point):
// (I - pmBeta L_y) du = Rhs ; u* = u + du written to the u* buffers.
// Block: TI consecutive i at one k, all j; threads = TI * P; blockIdx.z = component.
template <class T, int TI>
__global__ void __launch_bounds__(256) k_uhat_pimp(Geo<T> g, const double* __restrict__ fac, int P,
                                                   const T* __restrict__ ux, const T* __restrict__ uy,
                                                   const T* __restrict__ uz, const T* __restrict__ rx,
                                                   const T* __restrict__ ry, const T* __restrict__ rz,
                                                   T* __restrict__ uxs, T* __restrict__ uys, T* __restrict__ uzs,
                                                   const DevScalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int comp = blockIdx.z;
  const T* u = comp == 0 ? ux : (comp == 1 ? uy : uz);
  T* us = comp == 0 ? uxs : (comp == 1 ? uys : uzs);
  const T* rhs = comp == 0 ? rx : (comp == 1 ? ry : rz);
  const int nx = g.nx, ny = g.ny, k = blockIdx.y, i0 = blockIdx.x * TI, Q = P - 1;
  const double* F64 = fac + (size_t)(comp == 1 ? 1 : 0) * helm_set_stride(ny, P);
  const double *RM = F64, *AA = F64 + ny, *CP = F64 + 2 * ny, *AL = F64 + 3 * ny, *BE = F64 + 4 * ny,
               *IFD = F64 + 5 * ny;
  T* F = (T*)smem_raw;                    // ny * TI
  T* IF = F + (size_t)ny * TI;            // TI * 2Q
  // the 4th-order and FIMP RhsX already carry the forcing (k_rhs4, k_rhs_fimp)
  const T add = (comp == 0 && g.order != 4 && g.implicit != 2) ? (T)sc->dpmdxns : (T)0;
  const int tid = threadIdx.x;
  // the block's right-hand sides (coalesced rows of TI values) by asynchronous
  // copies, all in flight at once
  for (int t = tid; t < ny * TI; t += blockDim.x) {
    const int j = t / TI, ii = t % TI, i = i0 + ii;
    if (i < nx) cp_async_el(F + t, rhs + i + (long long)nx * (j + (long long)ny * k));
  }
  cp_async_commit();
  cp_async_wait<0>();  // this thread's copies (the slots it reads next)
  for (int t = tid; t < ny * TI; t += blockDim.x) {
    const int j = t / TI, ii = t % TI, i = i0 + ii;
    T f = (T)0;
    if (i < nx) f = F[t] + add;
    if (comp == 1 && j == 0) f = (T)0;  // duy_ym: uy_ym is constant (Update_uy_ym_CH)
    F[t] = f;
  }
  __syncthreads();
  for (int t = tid; t < TI * P; t += blockDim.x) {
    const int ii = t % TI, p = t / TI;
    const int s = chunk_lo(p, ny, P), e = chunk_hi(p, ny, P);
    T d = (T)0;
    for (int j = s; j <= e; ++j) {
      const T f = F[j * TI + ii];
      d = (j == s) ? f * (T)RM[j] : (f - (T)AA[j] * d) * (T)RM[j];
      F[j * TI + ii] = d;
    }
    for (int j = e - 1; j >= s; --j) {
      d = F[j * TI + ii] - (T)CP[j] * d;
      F[j * TI + ii] = d;
    }
  }
  __syncthreads();
  for (int t = tid; t < TI; t += blockDim.x) helm_interfaces<T>(IFD, F + t, TI, ny, P, IF + (size_t)t * 2 * (Q > 0 ? Q : 1));
  __syncthreads();
  for (int t = tid; t < ny * TI; t += blockDim.x) {
    const int j = t / TI, ii = t % TI, i = i0 + ii;
    if (i >= nx) continue;
    const int p = chunk_of(j, ny, P);
    const T* G = IF + (size_t)ii * 2 * (Q > 0 ? Q : 1);
    T x = F[t];
    if (p > 0) x += (T)AL[j] * G[2 * (p - 1)];
    if (p < P - 1) x += (T)BE[j] * G[2 * p + 1];
    const long long idx = i + (long long)nx * (j + (long long)ny * k);
    us[idx] = u[idx] + x;
  }
}

// ---------------------------------------------------------------------------
// clcPrSrcOther (src/CFD_2nd/m_TScheme.f90:213-241) fused with the forward
// x transform: src = div(u)/pmAlpha, packed as z_n = src_2n + i src_2n+1,
// complex FFT of length nx/2, then the real-to-complex split
// X_k = (Z_k + conj Z_{M-k})/2 - i W_nx^k (Z_k - conj Z_{M-k})/2, k = 0..M.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_prsrc_xfft(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                    const T* __restrict__ uy, const T* __restrict__ uz,
                                                    typename CplxOf<T>::type* __restrict__ spec, FFTPlanDev pl,
                                                    const typename CplxOf<T>::type* __restrict__ tw,
                                                    const typename CplxOf<T>::type* __restrict__ twr, int LPB, int mode,
                                                    DevScalars* __restrict__ sc, T* __restrict__ pr) {
  typedef typename CplxOf<T>::type CT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, M = nx / 2, nxh = g.nxh;
  const int nlines = ny * nz;
  const int line0 = blockIdx.x * LPB;
  const int nl = min(LPB, nlines - line0);
  CT* A = (CT*)smem_raw;
  CT* B = A + (size_t)LPB * M;
  const T sudtal = mode == 0 ? (T)(1.0 / sc->pmAlpha) : (T)1;
  const T rdx = g.rdx, rdz = g.rdz;
  double dmax = 0.0;
  for (int t = threadIdx.x; t < nl * M; t += blockDim.x) {
    const int l = t / M, n = t % M;
    const int line = line0 + l;
    const int j = line % ny, k = line / ny;
    const int kp = wrapp(k, nz);
    const int i0 = 2 * n, i1 = 2 * n + 1, i2 = wrapp(i1, nx);
    const long long base = (long long)nx * (j + (long long)ny * k);
    const T sucaj = m.rdyp[j + 1];
    const T u0 = ux[base + i0], u1 = ux[base + i1], u2 = ux[base + i2];
    const T v0 = uy[base + i0], v1 = uy[base + i1];
    const T v0p = fld(uy, g, 1, i0, j + 1, k), v1p = fld(uy, g, 1, i1, j + 1, k);
    const long long basep = (long long)nx * (j + (long long)ny * kp);
    const T w0 = uz[base + i0], w1 = uz[base + i1];
    const T w0p = uz[basep + i0], w1p = uz[basep + i1];
    T r0 = (u1 - u0) * rdx + (v0p - v0) * sucaj + (w0p - w0) * rdz;
    T r1 = (u2 - u1) * rdx + (v1p - v1) * sucaj + (w1p - w1) * rdz;
    if (g.order == 4) {
      const C4<T> c4(g);
      r0 = div4_cell(g, c4, sucaj, ux, uy, uz, i0, j, k);
      r1 = div4_cell(g, c4, sucaj, ux, uy, uz, i1, j, k);
    }
    if (mode == 2 || mode == 4) { r0 = u0; r1 = u1; }  // ux carries the source (standalone Poisson) or the field
    if (mode == 0 && g.implicit == 2) {     // clcPrSrc_FIMP: pressure += -xnu/2 div (m_TScheme.f90:271)
      const T xnuhm = -(T)0.5 * g.xnu;
      pr[base + i0] = pr[base + i0] + xnuhm * r0;
      pr[base + i1] = pr[base + i1] + xnuhm * r1;
    }
    dmax = fmax(dmax, fmax(fabs((double)r0), fabs((double)r1)));
    A[l * M + n] = mk(sudtal * r0, sudtal * r1);
  }
  // block max of |div| (any block size up to 1024)
  {
    __shared__ double wred[32];
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if ((threadIdx.x & 31) == 0) wred[threadIdx.x >> 5] = dmax;
    __syncthreads();
    if (threadIdx.x < 32) {
      double v = threadIdx.x < (blockDim.x + 31) / 32 ? wred[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (threadIdx.x == 0 && mode != 4) atomic_max_nonneg(&sc->divmax1, v);
    }
    __syncthreads();
  }
  const CT* Z = fft_lines<CT, false>(A, B, pl, nl, M, 1, tw);
  const T hf = (T)0.5;
  for (int t = threadIdx.x; t < nl * (M + 1); t += blockDim.x) {
    const int l = t / (M + 1), kk = t % (M + 1);
    const CT a = Z[l * M + (kk == M ? 0 : kk)];
    const CT b = cconj(Z[l * M + (kk == 0 ? 0 : M - kk)]);
    const CT e = mk(hf * (a.x + b.x), hf * (a.y + b.y));
    const CT dd = csub(a, b);
    const CT o = mk(hf * dd.y, -hf * dd.x);  // (a-b)/(2i)
    const CT w = __ldg(twr + kk);
    spec[(long long)nxh * (line0 + l) + kk] = cadd(e, cmul(w, o));
  }
}

// ---------------------------------------------------------------------------
// z transform of the spectrum, in place: layout (kx, j, kz), lines over kz.
// Block = TKX consecutive kx at one j; lines interleaved in shared memory.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_zfft(Geo<T> g, typename CplxOf<T>::type* __restrict__ spec, FFTPlanDev pl,
                                              const typename CplxOf<T>::type* __restrict__ tw, int TKX, int inverse,
                                              const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int nz = g.nz, ny = g.ny, nxh = g.nxh;
  const int kx0 = blockIdx.x * TKX, j = blockIdx.y;
  CT* A = (CT*)smem_raw;
  CT* B = A + (size_t)TKX * nz;
  const long long zs = (long long)nxh * ny;
  for (int t = threadIdx.x; t < TKX * nz; t += blockDim.x) {
    const int l = t % TKX, kz = t / TKX;
    const int kx = kx0 + l;
    CT v = mk((T)0, (T)0);
    if (kx < nxh) v = spec[kx + (long long)nxh * j + zs * kz];
    if (inverse) v = cconj(v);
    A[kz * TKX + l] = v;
  }
  __syncthreads();
  const CT* Z = fft_lines<CT, true>(A, B, pl, TKX, 1, TKX, tw);
  for (int t = threadIdx.x; t < TKX * nz; t += blockDim.x) {
    const int l = t % TKX, kz = t / TKX;
    const int kx = kx0 + l;
    if (kx >= nxh) continue;
    CT v = Z[kz * TKX + l];
    if (inverse) v = cconj(v);
    spec[kx + (long long)nxh * j + zs * kz] = v;
  }
}

// ---------------------------------------------------------------------------
// y tridiagonal per (kx,kz) (src/CFD_2nd/m_Poisson.f90:1114-1156):
// [am2Pr, ac2Pr + WaveNumX + WaveNumZ, ap2Pr], with the (kx,kz)=(0,0) system's
// first row replaced by the identity and zero right-hand side.  Solved in FP64
// in shared memory (also in the mixed path), partitioned as in k_uhat_pimp
// but with per-system factors.  Block = TS consecutive kx at one kz.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_ysolve(Geo<T> g, Metrics<double> m, const double* __restrict__ wave,
                                                typename CplxOf<T>::type* __restrict__ spec, int TS, int P,
                                                const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nxh = g.nxh;
  const int kx0 = blockIdx.x * TS, kz = blockIdx.y;
  const int Q = P - 1;
  double2* F = (double2*)smem_raw;               // ny * TS
  double* CP = (double*)(F + (size_t)ny * TS);   // ny * TS  (cp, later beta)
  double* AL = CP + (size_t)ny * TS;             // ny * TS
  double2* IFc = (double2*)(AL + (size_t)ny * TS); // TS * Q * 2
  double* RED = (double*)(IFc + (size_t)TS * (Q > 0 ? Q : 1) * 2);  // TS * Q * 5 : Minv(4), v
  const long long zs = (long long)nxh * ny;
  for (int t = threadIdx.x; t < ny * TS; t += blockDim.x) {
    const int s = t % TS, j = t / TS;
    const int kx = kx0 + s;
    double2 v = make_double2(0.0, 0.0);
    if (kx < nxh) {
      CT c = spec[kx + (long long)nxh * j + zs * kz];
      v = make_double2((double)c.x, (double)c.y);
    }
    F[t] = v;
  }
  __syncthreads();
  const double wz = wave[nx + kz];
  for (int t = threadIdx.x; t < TS * P; t += blockDim.x) {
    const int s = t % TS, p = t / TS;
    const int kx = kx0 + s;
    const double lam = wave[kx < nxh ? kx : 0] + wz;
    const bool pin = (kx == 0 && kz == 0);
    const int jlo = chunk_lo(p, ny, P), jhi = chunk_hi(p, ny, P);
    double cpp = 0.0, dal = 0.0;
    double2 d = make_double2(0.0, 0.0);
    for (int j = jlo; j <= jhi; ++j) {
      const int jc = j + 1;
      double a = m.am2Pr[jc], c = m.ap2Pr[jc], b = m.ac2Pr[jc] + lam;
      double2 f = F[j * TS + s];
      if (pin && j == 0) { a = 0.0; b = 1.0; c = 0.0; f = make_double2(0.0, 0.0); }
      const double mm = (j == jlo) ? b : b - a * cpp;
      const double rm = 1.0 / mm;
      const double cp = c * rm;
      if (j == jlo) { d.x = f.x * rm; d.y = f.y * rm; dal = -a * rm; }
      else { d.x = (f.x - a * d.x) * rm; d.y = (f.y - a * d.y) * rm; dal = -a * dal * rm; }
      F[j * TS + s] = d;
      CP[j * TS + s] = cp;
      AL[j * TS + s] = (p == 0) ? 0.0 : dal;
      cpp = cp;
    }
    double be = (p == P - 1) ? 0.0 : -CP[jhi * TS + s];
    double al = AL[jhi * TS + s];
    double2 y = F[jhi * TS + s];
    CP[jhi * TS + s] = be;
    for (int j = jhi - 1; j >= jlo; --j) {
      const double cp = CP[j * TS + s];
      const double2 dj = F[j * TS + s];
      y.x = dj.x - cp * y.x; y.y = dj.y - cp * y.y;
      al = AL[j * TS + s] - cp * al;
      be = -cp * be;
      F[j * TS + s] = y;
      AL[j * TS + s] = al;
      CP[j * TS + s] = be;
    }
  }
  __syncthreads();
  if (threadIdx.x < TS && Q > 0) {
    const int s = threadIdx.x;
    double* R = RED + (size_t)s * Q * 5;
    double2* G = IFc + (size_t)s * Q * 2;
    double m01p = 0.0, vprev = 0.0;
    double2 gu = make_double2(0.0, 0.0), gw;
    for (int q = 0; q < Q; ++q) {
      const int eq = chunk_hi(q, ny, P), sq1 = chunk_lo(q + 1, ny, P);
      const double l = -AL[eq * TS + s], v = -CP[sq1 * TS + s];
      double d00 = 1.0, d01 = -CP[eq * TS + s], d10 = -AL[sq1 * TS + s], d11 = 1.0;
      if (q > 0) d01 -= l * m01p * vprev;  // (L_q Minv_{q-1} U_{q-1}) has only a (0,1) entry
      const double r = 1.0 / (d00 * d11 - d01 * d10);
      const double M00 = d11 * r, M01 = -d01 * r, M10 = -d10 * r, M11 = d00 * r;
      double2 ru = F[eq * TS + s];
      if (q > 0) { ru.x -= l * gu.x; ru.y -= l * gu.y; }
      const double2 rw = F[sq1 * TS + s];
      gu = make_double2(M00 * ru.x + M01 * rw.x, M00 * ru.y + M01 * rw.y);
      gw = make_double2(M10 * ru.x + M11 * rw.x, M10 * ru.y + M11 * rw.y);
      G[2 * q] = gu; G[2 * q + 1] = gw;
      R[5 * q + 0] = M00; R[5 * q + 1] = M01; R[5 * q + 2] = M10; R[5 * q + 3] = M11; R[5 * q + 4] = v;
      m01p = M01; vprev = v;
    }
    double2 zw = G[2 * (Q - 1) + 1];
    for (int q = Q - 2; q >= 0; --q) {
      const double* Rq = R + 5 * q;
      const double fx = Rq[4] * zw.x, fy = Rq[4] * zw.y;
      double2 zu = G[2 * q], zwn = G[2 * q + 1];
      zu.x -= Rq[1] * fx; zu.y -= Rq[1] * fy;
      zwn.x -= Rq[3] * fx; zwn.y -= Rq[3] * fy;
      G[2 * q] = zu; G[2 * q + 1] = zwn;
      zw = zwn;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ny * TS; t += blockDim.x) {
    const int s = t % TS, j = t / TS;
    const int kx = kx0 + s;
    if (kx >= nxh) continue;
    const int p = chunk_of(j, ny, P);
    double2 x = F[t];
    const double2* G = IFc + (size_t)s * Q * 2;
    if (p > 0) { const double al = AL[t]; x.x += al * G[2 * (p - 1)].x; x.y += al * G[2 * (p - 1)].y; }
    if (p < P - 1) { const double be = CP[t]; x.x += be * G[2 * p + 1].x; x.y += be * G[2 * p + 1].y; }
    spec[kx + (long long)nxh * j + zs * kz] = mk((T)x.x, (T)x.y);
  }
}

// ---------------------------------------------------------------------------
// y solve with per-mode factors precomputed once per run (the Poisson matrix
// of mode (kx,kz) does not change during a run).  Factors depend on kz only
// through WaveNumZ, which is even in kz, so modes kz and nz-kz share them;
// the grid visits kz and nz-kz back to back so that the second read hits L2.
// Layout (FP64): RM[(kzh*ny + j)*nxh + kx], CP likewise (chunk-local LU),
// IFD[((kzh*Q + q)*6 + c)*nxh + kx] (interface block factors Minv, l, v).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int kz_of_block(int y, int nz) {
  return y == 0 ? 0 : ((y & 1) ? (y + 1) / 2 : nz - y / 2);
}

// Factors of the Thomas elimination of the Poisson y systems
// [am2Pr, ac2Pr + wx(kx) + wz(kz), ap2Pr] (src/CFD_2nd/m_Poisson.f90:1126-1150,
// InverseTridiagonal, m_Tools.f90:224-251), one thread per (kx, |kz|) column:
// rm_j = 1 / (b_j - a_j cp_{j-1}), cp_j = c_j rm_j; row 1 of the (0,0) system
// is replaced by phi = 0 (:1136-1140).  They depend on the grid only and are
// computed once per run, in FP64 and stored in precision R, layout
// ((kzh * ny) + j) * ldx + kx.
template <class R>
__global__ void __launch_bounds__(128) k_ythomas_factors(Metrics<double> m, const double* __restrict__ wave, int nx,
                                                         int ny, R* __restrict__ RMf, R* __restrict__ CPf, int ldx,
                                                         int kxn) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzh = blockIdx.y;
  if (kx >= kxn) return;
  const double lam = wave[kx] + wave[nx + kzh];
  const bool pin = (kx == 0 && kzh == 0);
  double cp = 0.0;
  for (int j = 0; j < ny; ++j) {
    const int jc = j + 1;
    double a = m.am2Pr[jc], c = m.ap2Pr[jc], b = m.ac2Pr[jc] + lam;
    if (pin && j == 0) { a = 0.0; b = 1.0; c = 0.0; }
    const double rm = 1.0 / (j == 0 ? b : b - a * cp);
    cp = c * rm;
    const size_t o = ((size_t)kzh * ny + j) * ldx + kx;
    RMf[o] = (R)rm;
    CPf[o] = (R)cp;
  }
}

template <class R> struct Vec2Of;
template <> struct Vec2Of<double> { typedef double2 type; };
template <> struct Vec2Of<float> { typedef float2 type; };

// Poisson y solve, Thomas across threads: one thread per (kx, kz) column,
// threads numbered kx fastest so that a warp reads 32 consecutive kx of one
// row of the (kx, j, kz) spectrum.  The forward sweep keeps d_j in place in
// the spectrum (the FP64 low modes of the mixed path in an FP64 scratch
// array, layout [j][low column]), the backward sweep overwrites it with the
// solution.  Rows are processed in batches of YB: the batch's loads are all
// issued before its dependent recurrence, so YB rows of every column are in
// flight at once.  YB is 16 in the FP64 kernel and 8 in the mixed one (whose
// FP64 low-mode sweeps share the FP32 sweeps' register budget); at 768x384x576
// the spectral group takes 2.51 ms FP64 with 16 rows against 2.61 with 8, mixed
// 1.65 with 8 against 1.73 with 16; refilling each row's slot as soon as it is
// consumed instead of whole batches was slower in both.

template <class R, class CT, int YB, class LD, class ST, class STD, class LDD>
__device__ __forceinline__ void thomas_column(int ny, bool pin, const R* __restrict__ rm, const R* __restrict__ cp,
                                              size_t fst, const double* __restrict__ am, LD load, ST store,
                                              STD store_d, LDD load_d) {
  R dx = (R)0, dy = (R)0;
  for (int j0 = 0; j0 < ny; j0 += YB) {
    R fx[YB], fy[YB], r[YB], a[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j < ny) {
        const CT f = load(j);
        fx[u] = (R)f.x; fy[u] = (R)f.y;
        r[u] = __ldg(rm + fst * j);
        a[u] = (R)__ldg(am + j + 1);
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j < ny) {
        if (j == 0) {
          dx = pin ? (R)0 : fx[u] * r[u];
          dy = pin ? (R)0 : fy[u] * r[u];
        } else {
          dx = (fx[u] - a[u] * dx) * r[u];
          dy = (fy[u] - a[u] * dy) * r[u];
        }
        store_d(j, dx, dy);
      }
    }
  }
  store(ny - 1, dx, dy);
  for (int j1 = ny - 2; j1 >= 0; j1 -= YB) {
    R ex[YB], ey[YB], c[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j1 - u;
      if (j >= 0) {
        const CT v = load_d(j);
        ex[u] = (R)v.x; ey[u] = (R)v.y;
        c[u] = __ldg(cp + fst * j);
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j1 - u;
      if (j >= 0) {
        dx = ex[u] - c[u] * dx;
        dy = ey[u] - c[u] * dy;
        store(j, dx, dy);
      }
    }
  }
}

// All columns in the precision of the field (FP64 path), or in the mixed
// path the FP32 columns: the low modes kx < KX, |kz| <= KL are skipped
// (KX = 0: none) and solved by k_ythomas_low.
template <class T, class R, int YB>
__global__ void __launch_bounds__(128) k_ythomas(Geo<T> g, Metrics<double> m, const R* __restrict__ RMf,
                                                 const R* __restrict__ CPf, typename CplxOf<T>::type* __restrict__ spec,
                                                 int KL, int KX, const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  if (sc->status) return;
  const int nxh = g.nxh, ny = g.ny, nz = g.nz;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nxh * nz) return;
  const int kx = (int)(t % nxh), kz = (int)(t / nxh);
  const int kzh = kz <= nz - kz ? kz : nz - kz;
  if (kx < KX && kzh <= KL) return;
  const size_t st = (size_t)nxh;
  CT* col = spec + kx + st * ny * kz;
  const R* rm = RMf + (size_t)kzh * ny * st + kx;
  const R* cp = CPf + (size_t)kzh * ny * st + kx;
  auto load = [&](int j) { return col[st * j]; };
  auto store = [&](int j, R x, R y) { col[st * j] = mk((T)x, (T)y); };
  thomas_column<R, CT, YB>(ny, kx == 0 && kz == 0, rm, cp, st, m.am2Pr, load, store, store, load);
}

// Mixed path: the low modes kx < KX, |kz| <= KL (column zi = kz for kz <= KL,
// KL + nz - kz above) in FP64 with FP64 factors, their forward sweep kept in
// the FP64 scratch [j][low column].
template <class T>
__global__ void __launch_bounds__(128) k_ythomas_low(Geo<T> g, Metrics<double> m, const double* __restrict__ RM64,
                                                     const double* __restrict__ CP64,
                                                     typename CplxOf<T>::type* __restrict__ spec,
                                                     double2* __restrict__ scr, int KL, int KX,
                                                     const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  if (sc->status) return;
  const int nxh = g.nxh, ny = g.ny, nz = g.nz;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (2 * KL + 1) * KX) return;
  const int zi = q / KX, kx = q - zi * KX;
  const int kz = zi <= KL ? zi : nz - (zi - KL);
  if (kx >= nxh || (zi > KL && kz <= KL)) return;
  const int kzh = kz <= nz - kz ? kz : nz - kz;
  const size_t st = (size_t)nxh;
  CT* col = spec + kx + st * ny * kz;
  const size_t nlow = (size_t)(2 * KL + 1) * KX;
  double2* w = scr + (size_t)zi * KX + kx;  // [j][low column]
  auto load = [&](int j) { const CT v = col[st * j]; return make_double2(v.x, v.y); };
  auto store = [&](int j, double x, double y) { col[st * j] = mk((T)x, (T)y); };
  auto store_d = [&](int j, double x, double y) { w[nlow * j] = make_double2(x, y); };
  auto load_d = [&](int j) { return w[nlow * j]; };
  thomas_column<double, double2, 16>(ny, kx == 0 && kz == 0, RM64 + (size_t)kzh * ny * KX + kx,
                                     CP64 + (size_t)kzh * ny * KX + kx, (size_t)KX, m.am2Pr, load, store, store_d,
                                     load_d);
}

// ---------------------------------------------------------------------------
// Periodic y (clcPPE_z1_periodic, src/CFD_2nd/m_Poisson.f90:954-1073): the
// systems [am2Pr, ac2Pr + wx(kx) + wz(kz), ap2Pr] are cyclic, solved by
// InversePeriodicTridiagonal (src/CFD_2nd/m_Tools.f90:109-162), with row 1
// of the (0,0) system replaced by phi = 0 (:1012-1029).  Its coefficient
// recurrences depend on the mode only and are computed once per run, one
// thread per (kx, |kz|), FP64, layout ((kzh * ny) + j) * nxh + kx:
//   PP_0 = b_1 (row 1 divides), PP_j = 1 / (b + a arrmn1_{j-1}) (ppj),
//   A1_j = arrmn1_j, A1_{n-1} = the closing denominator,
//   A2_j = arrmn2_j after the backward pass.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_ycyclic_factors(Metrics<double> m, const double* __restrict__ wave, int nx,
                                                         int ny, int nxh, double* __restrict__ PP,
                                                         double* __restrict__ A1, double* __restrict__ A2) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzh = blockIdx.y;
  if (kx >= nxh) return;
  const double lam = wave[kx] + wave[nx + kzh];
  const bool pin = (kx == 0 && kzh == 0);
  const size_t st = (size_t)nxh, o = (size_t)kzh * ny * st + kx;
  auto coef = [&](int j, double& a, double& b, double& c) {
    a = m.am2Pr[j + 1]; c = m.ap2Pr[j + 1]; b = m.ac2Pr[j + 1] + lam;
    if (pin && j == 0) { a = 0.0; b = 1.0; c = 0.0; }
  };
  double a, b, c;
  coef(0, a, b, c);
  double v1 = -c / b, v2 = -a / b;
  PP[o] = b; A1[o] = v1; A2[o] = v2;
  for (int j = 1; j <= ny - 2; ++j) {
    coef(j, a, b, c);
    const double ppj = 1.0 / (b + a * v1);
    v1 = -c * ppj;
    v2 = -a * v2 * ppj;
    PP[o + st * j] = ppj; A1[o + st * j] = v1; A2[o + st * j] = v2;
  }
  // backward pass: arrmn2_n = 1, arrmn2_j += arrmn1_j arrmn2_{j+1}
  double w = 1.0;
  A2[o + st * (ny - 1)] = w;
  for (int j = ny - 2; j >= 0; --j) {
    w = A2[o + st * j] + A1[o + st * j] * w;
    A2[o + st * j] = w;
  }
  coef(ny - 1, a, b, c);
  A1[o + st * (ny - 1)] = c * A2[o] + a * A2[o + st * (ny - 2)] + b;
}

// One thread per (kx, kz) column of the (kx, j, kz) spectrum (kx fastest, so
// a warp reads 32 consecutive kx of one row), FP64, in place: forward
// elimination, the backward pass of the right-hand side (arrmn3), the closure
// of row n, and the back substitution f_j = f_n arrmn2_j + arrmn3_j.  Each
// pass loads YB rows (and their factors) before its dependent recurrence, so
// YB loads of every column are in flight at once.
template <class T, int YB>
__global__ void __launch_bounds__(128) k_ycyclic(Geo<T> g, Metrics<double> m, const double* __restrict__ PP,
                                                 const double* __restrict__ A1, const double* __restrict__ A2,
                                                 typename CplxOf<T>::type* __restrict__ spec,
                                                 const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  if (sc->status) return;
  const int nxh = g.nxh, ny = g.ny, nz = g.nz;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nxh * nz) return;
  const int kx = (int)(t % nxh), kz = (int)(t / nxh);
  const int kzh = kz <= nz - kz ? kz : nz - kz;
  const size_t st = (size_t)nxh;
  CT* col = spec + kx + st * ny * kz;
  const size_t o = (size_t)kzh * ny * st + kx;
  const bool pin = (kx == 0 && kz == 0);
  // forward elimination, rows 1..n-1 (0-based 0..ny-2); row 1 divides by b_1
  double dx = 0.0, dy = 0.0;
  for (int j0 = 0; j0 <= ny - 2; j0 += YB) {
    double fx[YB], fy[YB], pp[YB], am[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j <= ny - 2) {
        const CT f = col[st * j];
        fx[u] = (double)f.x; fy[u] = (double)f.y;
        pp[u] = PP[o + st * j];
        am[u] = m.am2Pr[j + 1];
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j <= ny - 2) {
        if (j == 0) {
          dx = pin ? 0.0 : fx[u] / pp[u];
          dy = pin ? 0.0 : fy[u] / pp[u];
        } else {
          dx = (fx[u] - am[u] * dx) * pp[u];
          dy = (fy[u] - am[u] * dy) * pp[u];
        }
        col[st * j] = mk((T)dx, (T)dy);
      }
    }
  }
  // backward pass: arrmn3_n = 0, arrmn3_j = f_j + arrmn1_j arrmn3_{j+1}
  double ex = 0.0, ey = 0.0, lx = 0.0, ly = 0.0;
  for (int j1 = ny - 2; j1 >= 0; j1 -= YB) {
    double vx[YB], vy[YB], a1[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j1 - u;
      if (j >= 0) {
        const CT f = col[st * j];
        vx[u] = (double)f.x; vy[u] = (double)f.y;
        a1[u] = A1[o + st * j];
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j1 - u;
      if (j >= 0) {
        ex = vx[u] + a1[u] * ex;
        ey = vy[u] + a1[u] * ey;
        col[st * j] = mk((T)ex, (T)ey);
        if (j == ny - 2) { lx = ex; ly = ey; }
      }
    }
  }
  // closure of row n, then f_j = f_n arrmn2_j + arrmn3_j
  const double an = m.am2Pr[ny], cn = m.ap2Pr[ny], den = A1[o + st * (ny - 1)];
  const CT fl = col[st * (ny - 1)];
  const double fnx = ((double)fl.x - cn * ex - an * lx) / den, fny = ((double)fl.y - cn * ey - an * ly) / den;
  col[st * (ny - 1)] = mk((T)fnx, (T)fny);
  for (int j0 = 0; j0 <= ny - 2; j0 += YB) {
    double vx[YB], vy[YB], a2[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j <= ny - 2) {
        const CT f = col[st * j];
        vx[u] = (double)f.x; vy[u] = (double)f.y;
        a2[u] = A2[o + st * j];
      }
    }
#pragma unroll
    for (int u = 0; u < YB; ++u) {
      const int j = j0 + u;
      if (j <= ny - 2) col[st * j] = mk((T)(fnx * a2[u] + vx[u]), (T)(fny * a2[u] + vy[u]));
    }
  }
}

// ---------------------------------------------------------------------------
// inverse x transform (complex-to-real, unnormalised as FFTW's HC2R) * normfft
// (src/CFD_2nd/m_Poisson.f90:1194-1200) -> phi.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_xifft(Geo<T> g, const typename CplxOf<T>::type* __restrict__ spec,
                                               T* __restrict__ phi, FFTPlanDev pl,
                                               const typename CplxOf<T>::type* __restrict__ tw,
                                               const typename CplxOf<T>::type* __restrict__ twr, int LPB, T normfft,
                                               const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, M = nx / 2, nxh = g.nxh;
  const int nlines = ny * nz;
  const int line0 = blockIdx.x * LPB;
  const int nl = min(LPB, nlines - line0);
  CT* A = (CT*)smem_raw;
  CT* B = A + (size_t)LPB * M;
  for (int t = threadIdx.x; t < nl * M; t += blockDim.x) {
    const int l = t / M, kk = t % M;
    const CT* X = spec + (long long)nxh * (line0 + l);
    const CT a = X[kk];
    const CT b = cconj(X[M - kk]);
    const CT e = cadd(a, b);
    const CT o = cmul(csub(a, b), cconj(__ldg(twr + kk)));
    // Z_k = e + i o ; stored conjugated for the forward-transform-based inverse
    const CT z = mk(e.x - o.y, e.y + o.x);
    A[l * M + kk] = cconj(z);
  }
  __syncthreads();
  const CT* Z = fft_lines<CT, false>(A, B, pl, nl, M, 1, tw);
  for (int t = threadIdx.x; t < nl * M; t += blockDim.x) {
    const int l = t / M, n = t % M;
    const CT z = cconj(Z[l * M + n]);
    const long long base = (long long)nx * (line0 + l);
    phi[base + 2 * n] = z.x * normfft;
    phi[base + 2 * n + 1] = z.y * normfft;
  }
}

// Block reductions of a 256-thread block with warp shuffles: the result is
// valid in thread 0 (order of the sums fixed, so results are reproducible).
__device__ __forceinline__ double block_sum256(double v, double* sh /* 8 */) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int tl = threadIdx.x + blockDim.x * threadIdx.y;
  if ((tl & 31) == 0) sh[tl >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (tl == 0)
    for (int w = 0; w < 8; ++w) r += sh[w];
  return r;
}
__device__ __forceinline__ double block_max256(double v, double* sh /* 8 */) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tl = threadIdx.x + blockDim.x * threadIdx.y;
  if ((tl & 31) == 0) sh[tl >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (tl == 0)
    for (int w = 0; w < 8; ++w) r = fmax(r, sh[w]);
  return r;
}

// ---------------------------------------------------------------------------
// FluidVelUpdate (src/CFD_2nd/m_TScheme.f90:281-306) + PressureUpdate_PIMP
// (src/CFD_2nd/m_TSchemePIMP_inc.f90:852-873), phi ghosts from
// SetBC_and_UpdateHalo_pr (Neumann in y, periodic x,z), plus the block partial
// sums of ux*dyp used by the next substep's bulk constraint.
// mode 1: projection only (pmAlpha = 1, no pressure update).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_proj(Geo<T> g, Metrics<T> m, const T* uxs, const T* uys, const T* uzs,
                                              T* ux, T* uy, T* uz, T* __restrict__ pr, const T* __restrict__ phi,
                                              double* __restrict__ part, int mode, const DevScalars* __restrict__ sc,
                                              const T* __restrict__ nut) {
  __shared__ double red[8];
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tl = threadIdx.x + blockDim.x * threadIdx.y;
  double s = 0.0;
  if (i < nx && j < ny) {
    const int jc = j + 1;
    const int im = wrapm(i, nx), km = wrapm(k, nz);
    const long long idx = i + (long long)nx * (j + (long long)ny * k);
    const T pmAlpha = mode == 0 ? (T)sc->pmAlpha : (T)1;
    const T phic = phi[idx];
    const T phim_x = phi[im + (long long)nx * (j + (long long)ny * k)];
    const int jm = j > 0 ? j - 1 : (g.bc.lo == 0 ? ny - 1 : 0);  // phi(ic,0,kc): Neumann or periodic halo
    const T phim_y = phi[i + (long long)nx * (jm + (long long)ny * k)];
    const T phim_z = phi[i + (long long)nx * (j + (long long)ny * km)];
    const T rdxEta2 = g.rdx * pmAlpha, rdzEta2 = g.rdz * pmAlpha, sucacEta2 = m.rdyc[jc] * pmAlpha;
    T uxn = uxs[idx] - (phic - phim_x) * rdxEta2;
    T uyn = uys[idx] - (phic - phim_y) * sucacEta2;
    T uzn = uzs[idx] - (phic - phim_z) * rdzEta2;
    if (g.order == 4) {  // FluidVelUpdate, src/CFD_4th/m_TScheme.f90:148-173
      const C4<T> c4(g);
      const Nbr n = make_nbr(g, i, j, k);
      const T dpdx = c4.dx1 * at(phi, n, n.xm2) + c4.dx2 * phim_x + c4.dx3 * phic + c4.dx4 * at(phi, n, n.xp);
      const T dpdy = (phic - phim_y) * m.rdyc[jc];
      const T dpdz = c4.dz1 * at(phi, n, n.zm2) + c4.dz2 * phim_z + c4.dz3 * phic + c4.dz4 * at(phi, n, n.zp);
      uxn = uxs[idx] - pmAlpha * dpdx;
      uyn = uys[idx] - pmAlpha * dpdy;
      uzn = uzs[idx] - pmAlpha * dpdz;
    }
    ux[idx] = uxn;
    uy[idx] = uyn;
    uz[idx] = uzn;
    if (mode == 0 && g.les && g.implicit == 1) {  // PressureUpdate_PIMP_LES (src/CFD_2nd/m_TSchemePIMP_inc.f90:878-904)
      const T phip_y = phi[i + (long long)nx * ((j < ny - 1 ? j + 1 : ny - 1) + (long long)ny * k)];
      const T nc = nut[idx];
      const T njp = j < ny - 1 ? nut[idx + nx] : (g.bc.hi == -1 ? (T)2 * g.xnu - nc : nc);
      const T njm = j > 0 ? nut[idx - nx] : (g.bc.lo == -1 ? (T)2 * g.xnu - nc : nc);
      const T pmBetaT = (T)sc->pmBetaT;
      const T metr1 = m.rdyp[jc] * m.rdyc[jc], metr2 = m.rdyp[jc] * m.rdyc[jc + 1];
      const T visd = (T)0.5 * (njp + nc), visc = (T)0.5 * (nc + njm);
      const T pmBetap = -pmBetaT * metr2 * visd;
      const T pmBetam = -pmBetaT * metr1 * visc;
      const T pmBetac = -(pmBetap + pmBetam) + (T)1;
      pr[idx] = pr[idx] + pmBetap * phip_y + pmBetac * phic + pmBetam * phim_y;
    } else if (mode == 0 && (g.implicit == 2 || g.implicit == 0)) {
      // PressureUpdate_FIMP (src/CFD_2nd/m_TSchemeFIMP_inc.f90:1371-1386), _FEXP and
      // _FEXP_LES (src/CFD_2nd/m_TSchemeFEXP_inc.f90:513-548)
      pr[idx] = pr[idx] + phic;
    } else if (mode == 0) {
      const int jp = j < ny - 1 ? j + 1 : (g.bc.hi == 0 ? 0 : ny - 1);  // phi(ic,nyp,kc): Neumann or periodic halo
      const T phip_y = phi[i + (long long)nx * (jp + (long long)ny * k)];
      const T pmBeta = (T)sc->pmBeta;
      const T pmBetap = -pmBeta * m.ap2Pr[jc];
      const T pmBetac = -pmBeta * m.ac2Pr[jc] + (T)1;
      const T pmBetam = -pmBeta * m.am2Pr[jc];
      pr[idx] = pr[idx] + pmBetap * phip_y + pmBetac * phic + pmBetam * phim_y;
    }
    s = (double)uxn * (double)m.s1coe[jc];
  }
  const double bs = block_sum256(s, red);
  if (tl == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = bs;
}

// bulk partial sums of ux*s1coe for a freshly uploaded field
template <class T>
__global__ void __launch_bounds__(256) k_bulk_partial(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                      double* __restrict__ part) {
  __shared__ double red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int tl = threadIdx.x + blockDim.x * threadIdx.y;
  double s = 0.0;
  if (i < g.nx && j < g.ny) s = (double)ux[i + (long long)g.nx * (j + (long long)g.ny * k)] * (double)m.s1coe[j + 1];
  red[tl] = s;
  __syncthreads();
  for (int w = blockDim.x * blockDim.y / 2; w > 0; w >>= 1) {
    if (tl < w) red[tl] += red[tl + w];
    __syncthreads();
  }
  if (tl == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = red[0];
}

// CheckDivergence, CalcVmax, CalcMaxCFL of the next step, CalcUxAver partials
// (src/CFD_2nd/m_Tools.f90:21-104,250-270).  A thread walks `rows` rows of
// one (i, k) column (uy(j+1) carried to the next row), a block of 32 x 4
// columns reduces its maxima and sum and issues one atomic per quantity
// (per-cell blocks made the same-address atomics the bottleneck).
template <class T>
__global__ void __launch_bounds__(128) k_diag(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                              const T* __restrict__ uy, const T* __restrict__ uz,
                                              double* __restrict__ part, DevScalars* __restrict__ sc, int rows) {
  __shared__ double red[6][4];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  const int j0 = blockIdx.z * rows, j1 = min(j0 + rows, ny);
  double dv = 0, v0 = 0, v1 = 0, v2 = 0, cf = 0, s = 0;
  if (i < nx && k < nz) {
    const long long plane = (long long)nx * ny;
    const long long col = i + plane * k;
    const long long dxp = i + 1 == nx ? 1 - nx : 1;
    const long long dzp = k + 1 == nz ? -(long long)(nz - 1) * plane : plane;
    const double rdx = g.rdx, rdz = g.rdz;
    double b = uy[col + (long long)j0 * nx];
    const C4<T> c4(g);
    Nbr n4 = make_nbr(g, i, j0, k);  // the 4th-order divergence's neighbourhood, moved up row by row
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
      if (j > j0) nbr_next_row(n4, g, j);
      const long long idx = col + (long long)j * nx;
      const int jc = j + 1;
      const double a = ux[idx], c = uz[idx];
      const double aip = ux[idx + dxp], ckp = uz[idx + dzp];
      const double bjp = j + 1 < ny ? (double)uy[idx + nx]
                                    : (g.bc.hi == 0 ? (double)uy[col] : (double)(T)g.bc.uy_hi);  // periodic: row 0
      const double rdyp = m.rdyp[jc];
      double d = fabs((aip - a) * rdx + (bjp - b) * rdyp + (ckp - c) * rdz);
      if (g.order == 4) d = fabs((double)div4_at(g, c4, m.rdyp[jc], ux, uy, uz, n4));
      // fmax(NaN, x) = x on the device, so NaN is folded into +inf first: a NaN
      // field still trips the limit checks of the step
      if (!(d == d)) d = INFINITY;
      dv = fmax(dv, d);
      v0 = fmax(v0, a == a ? fabs(a) : INFINITY);
      v1 = fmax(v1, b == b ? fabs(b) : INFINITY);
      v2 = fmax(v2, c == c ? fabs(c) : INFINITY);
      cf = fmax(cf, fabs(a + aip) * rdx + fabs(b + bjp) * rdyp + fabs(c + ckp) * rdz);
      s += a * (double)m.dyp[jc];
      b = bjp;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    dv = fmax(dv, __shfl_xor_sync(0xffffffffu, dv, o));
    v0 = fmax(v0, __shfl_xor_sync(0xffffffffu, v0, o));
    v1 = fmax(v1, __shfl_xor_sync(0xffffffffu, v1, o));
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
    cf = fmax(cf, __shfl_xor_sync(0xffffffffu, cf, o));
    s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = cf; red[1][w] = dv; red[2][w] = v0; red[3][w] = v1; red[4][w] = v2; red[5][w] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[6];
    for (int q = 0; q < 5; ++q) r[q] = fmax(fmax(red[q][0], red[q][1]), fmax(red[q][2], red[q][3]));
    r[5] = (red[5][0] + red[5][1]) + (red[5][2] + red[5][3]);
    atomic_max_nonneg(&sc->uddx, r[0] * 0.5);
    atomic_max_nonneg(&sc->divmax2, r[1]);
    atomic_max_nonneg(&sc->vmax[0], r[2]);
    atomic_max_nonneg(&sc->vmax[1], r[3]);
    atomic_max_nonneg(&sc->vmax[2], r[4]);
    part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = r[5];
  }
}

__global__ void k_diag_reset(DevScalars* sc) {
  if (sc->status) return;
  sc->divmax2 = 0ull; sc->vmax[0] = 0ull; sc->vmax[1] = 0ull; sc->vmax[2] = 0ull; sc->uddx = 0ull;
}

// max |div u| of the current field into *slot (for ch3d_project)
template <class T>
__global__ void __launch_bounds__(256) k_divmax(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                const T* __restrict__ uy, const T* __restrict__ uz,
                                                unsigned long long* slot) {
  __shared__ double red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int tl = threadIdx.x + blockDim.x * threadIdx.y;
  double dv = 0;
  if (i < g.nx && j < g.ny) {
    const int ip = wrapp(i, g.nx), kp = wrapp(k, g.nz);
    const long long idx = i + (long long)g.nx * (j + (long long)g.ny * k);
    dv = fabs(((double)ux[ip + (long long)g.nx * (j + (long long)g.ny * k)] - ux[idx]) * g.rdx +
              ((double)fld(uy, g, 1, i, j + 1, k) - uy[idx]) * m.rdyp[j + 1] +
              ((double)uz[i + (long long)g.nx * (j + (long long)g.ny * kp)] - uz[idx]) * g.rdz);
    if (g.order == 4) dv = fabs((double)div4_cell(g, C4<T>(g), m.rdyp[j + 1], ux, uy, uz, i, j, k));
  }
  red[tl] = dv;
  __syncthreads();
  for (int w = blockDim.x * blockDim.y / 2; w > 0; w >>= 1) {
    if (tl < w) red[tl] = fmax(red[tl], red[tl + w]);
    __syncthreads();
  }
  if (tl == 0) atomic_max_nonneg(slot, red[0]);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static dim3 cell_grid(const ch3d_ctx* c) { return dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz); }
static dim3 cell_block() { return dim3(32, 8, 1); }


cudaError_t launch_step_begin(ch3d_ctx* c) {
  k_step_begin<<<1, 1, 0, c->stream>>>(c->sc, c->cfg.iCFL, c->cfg.CFLc, c->cfg.dtMax);
  return cudaGetLastError();
}

// first level of the deterministic two-level sum of block partials
__global__ void __launch_bounds__(256) k_reduce_partials(const double* __restrict__ in, int n, double* __restrict__ out) {
  __shared__ double red[256];
  const int nb = gridDim.x;
  const int chunk = (n + nb - 1) / nb;
  const int lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
  double s = 0.0;
  for (int q = lo + threadIdx.x; q < hi; q += blockDim.x) s += in[q];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

cudaError_t launch_reduce_partials(ch3d_ctx* c, const double* in, int n, double* out) {
  k_reduce_partials<<<CH3D_NRED, 256, 0, c->stream>>>(in, n, out);
  return cudaGetLastError();
}

cudaError_t launch_substep_setup(ch3d_ctx* c, int ns) {
  // the partials of the bulk sums (march projection or k_bulk_partial), or of the
  // 4th-order viscous sum (k_visc4_partial)
  const int np = c->cfg.order == 4 ? visc4_npart(c) : (c->march ? c->npart_m : c->npart);
  k_reduce_partials<<<CH3D_NRED, 256, 0, c->stream>>>(c->part, np, c->red1);
  const double norm_bulk = 1.0 / ((double)c->nx * (double)c->nz) / (c->cfg.ybulk2 - c->cfg.ybulk1);
  k_substep_setup<<<1, 256, 0, c->stream>>>(c->sc, c->red1, CH3D_NRED, ns, c->gam[ns - 1], c->the[ns - 1],
                                            c->alp[ns - 1], c->cfg.xnu, c->cfg.IsUxConst, c->cfg.ubulk, norm_bulk,
                                            c->cfg.order, (double)(c->nx * c->nz), c->cfg.yly);
  return cudaGetLastError();
}

cudaError_t launch_step_end(ch3d_ctx* c) {
  const double norm = 1.0 / ((double)c->nx * (double)c->nz) / c->cfg.yly;
  // part2: written by the fused projection (march layout) or by k_diag
  k_reduce_partials<<<CH3D_NRED, 256, 0, c->stream>>>(c->part2, march_diag_fusable(c) ? c->npart_m : diag_npart(c),
                                                       c->red2);
  k_step_end<<<1, 256, 0, c->stream>>>(c->sc, c->red2, CH3D_NRED, norm, c->cfg.div_limit, c->cfg.vel_limit);
  return cudaGetLastError();
}

template <class T> static cudaError_t rhs_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  k_rhs_pimp<T><<<cell_grid(c), cell_block(), 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], f[1], f[2], f[3],
                                                              f[4], f[5], f[6], f[7], f[8], f[9], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_rhs(ch3d_ctx* c) { return c->fp32 ? rhs_t<float>(c) : rhs_t<double>(c); }
template <class T> static cudaError_t rhs_fimp_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  const dim3 grid((c->nx + 31) / 32, (c->ny + 7) / 8, 3 * c->nz);  // z: component * nz + k
  k_rhs_fimp<T><<<grid, cell_block(), 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], f[1], f[2], f[3],
                                                              f[4], f[5], f[6], f[7], f[8], f[9], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_rhs_fimp(ch3d_ctx* c) { return c->fp32 ? rhs_fimp_t<float>(c) : rhs_fimp_t<double>(c); }

// clcU1/2/3Hat_FEXP (src/CFD_2nd/m_TSchemeFEXP_inc.f90:391-488): u* = u + Rhs,
// every cell; between walls the uy row on the lower wall then takes uy_ym,
// as SetBC_and_UpdateHaloForPrSrc (src/CFD_2nd/m_BC_and_Halo.f90:349-405)
// sets it before the divergence.  blockIdx.y = component.
template <class T>
__global__ void __launch_bounds__(256) k_uhat_fexp(Geo<T> g, const T* __restrict__ ux, const T* __restrict__ uy,
                                                   const T* __restrict__ uz, const T* __restrict__ rx,
                                                   const T* __restrict__ ry, const T* __restrict__ rz,
                                                   T* __restrict__ sx, T* __restrict__ sy, T* __restrict__ sz,
                                                   const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int comp = blockIdx.y;
  const T* u = comp == 0 ? ux : (comp == 1 ? uy : uz);
  const T* r = comp == 0 ? rx : (comp == 1 ? ry : rz);
  T* us = comp == 0 ? sx : (comp == 1 ? sy : sz);
  const long long plane = (long long)g.nx * g.ny;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < g.N; q += (long long)gridDim.x * blockDim.x) {
    T v = u[q] + r[q];
    if (comp == 1 && g.bc.lo != 0 && q % plane < g.nx) v = (T)g.bc.uy_lo;
    us[q] = v;
  }
}
template <class T> static cudaError_t uhat_fexp_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  const long long nb = (c->N + 255) / 256;
  const unsigned gx = (unsigned)(nb < 148LL * 16 ? nb : 148LL * 16);
  k_uhat_fexp<T><<<dim3(gx, 3), 256, 0, c->stream>>>(make_geo<T>(c), f[0], f[1], f[2], f[7], f[8], f[9], f[12], f[13],
                                                     f[14], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_uhat_fexp(ch3d_ctx* c) { return c->fp32 ? uhat_fexp_t<float>(c) : uhat_fexp_t<double>(c); }

cudaError_t launch_helm_factors(ch3d_ctx* c) {
  k_helm_factors<<<2, 64, 0, c->stream>>>(helm_coef(c), c->ny, c->Pv, c->hfac, c->sc);
  return cudaGetLastError();
}

template <class T> static cudaError_t uhat_t(ch3d_ctx* c) {
  constexpr int TI = 16;
  T** f = (T**)c->f;
  const int P = c->Pv, Q = P - 1;
  size_t smem = (size_t)c->ny * TI * sizeof(T) + (size_t)TI * 2 * (Q > 0 ? Q : 1) * sizeof(T) + 16;
  static PerDevice attr;  // per precision (template instance)
  auto kern = k_uhat_pimp<T, TI>;
  cudaError_t e = smem_limit_once(attr, c->device, kern, 200 * 1024);
  if (e != cudaSuccess) return e;
  dim3 grid((c->nx + TI - 1) / TI, c->nz, 3);
  int nthr = TI * P < 64 ? 64 : (TI * P > 256 ? 256 : TI * P);
  kern<<<grid, nthr, smem, c->stream>>>(make_geo<T>(c), c->hfac, P, f[0], f[1], f[2], f[7], f[8], f[9], f[12], f[13],
                                        f[14], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_uhat(ch3d_ctx* c) { return c->fp32 ? uhat_t<float>(c) : uhat_t<double>(c); }


// Shared-memory budget of one FFT block (two ping-pong buffers): three
// blocks of 256 threads fit in an SM.
static const int kFFTSmem = 74 * 1024;

template <class T> static int lines_per_block(int M) {
  int lpb = kFFTSmem / (2 * M * (int)sizeof(typename CplxOf<T>::type));
  if (lpb > 16) lpb = 16;
  if (lpb < 1) lpb = 1;
  return lpb;
}

template <class T> static cudaError_t prsrc_t(ch3d_ctx* c, int mode) {
  typedef typename CplxOf<T>::type CT;
  cudaError_t e;
  if (launch_prsrc_xfft_r(c, mode, &e)) return e;  // register FFT when the length has a plan
  T** f = (T**)c->f;
  const int M = c->nx / 2;
  const int LPB = lines_per_block<T>(M);
  const int nlines = c->ny * c->nz;
  size_t smem = (size_t)2 * LPB * M * sizeof(CT);
  static PerDevice attr;  // per precision (template instance)
  if ((e = smem_limit_once(attr, c->device, k_prsrc_xfft<T>, 200 * 1024)) != cudaSuccess) return e;
  const int nthr = 256;
  T* a = mode == 2 || mode == 4 ? f[10] : (mode == 1 ? f[0] : f[12]);
  T* b = mode == 1 ? f[1] : f[13];
  T* cz = mode == 1 ? f[2] : f[14];
  k_prsrc_xfft<T><<<(nlines + LPB - 1) / LPB, nthr, smem, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), a, b, cz,
                                                                      (CT*)c->spec, c->planx, (const CT*)c->twx,
                                                                      (const CT*)c->twr, LPB, mode, c->sc, f[3]);
  return cudaGetLastError();
}
cudaError_t launch_prsrc_xfft(ch3d_ctx* c, int mode) { return c->fp32 ? prsrc_t<float>(c, mode) : prsrc_t<double>(c, mode); }

template <class T> static cudaError_t spectral_t(ch3d_ctx* c) {
  typedef typename CplxOf<T>::type CT;
  const int nz = c->nz;
  cudaError_t e;
  const bool zr = launch_zfft_r(c, 0, &e);  // register FFT when nz has a plan
  if (zr && e != cudaSuccess) return e;
  int TKX = kFFTSmem / (2 * nz * (int)sizeof(CT));
  int t = 1;
  while (t * 2 <= TKX && t * 2 <= 16) t *= 2;
  TKX = t;
  size_t smemz = (size_t)2 * TKX * nz * sizeof(CT);
  const int nthrz = 256;
  static PerDevice attr;  // per precision (template instance)
  if ((e = smem_limit_once(attr, c->device, k_zfft<T>, 200 * 1024)) != cudaSuccess) return e;
  dim3 gz((c->nxh + TKX - 1) / TKX, c->ny);
  if (!zr) {
    k_zfft<T><<<gz, nthrz, smemz, c->stream>>>(make_geo<T>(c), (CT*)c->spec, c->planz, (const CT*)c->twz, TKX, 0, c->sc);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const unsigned gy = (unsigned)(((long long)c->nxh * c->nz + 127) / 128);
  if (y_periodic(c)) {  // periodic y (FP64 only): the cyclic systems
    k_ycyclic<T, 16><<<gy, 128, 0, c->stream>>>(make_geo<T>(c), c->m64full, (const double*)c->yRM,
                                                (const double*)c->yCP, c->yA2, (CT*)c->spec, c->sc);
  } else if (!c->fp32) {
    k_ythomas<T, double, 16><<<gy, 128, 0, c->stream>>>(make_geo<T>(c), c->m64full, (const double*)c->yRM,
                                                        (const double*)c->yCP, (CT*)c->spec, 0, 0, c->sc);
  } else {
    // mixed: FP32 systems and factors; the low modes near kx = kz = 0 in FP64 on the
    // high-priority side stream, overlapping the FP32 sweeps (a fork and a join in
    // the captured step graph)
    const int nlow = (2 * c->KL + 1) * c->TSy;
    if ((e = cudaEventRecord(c->ev_fork, c->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(c->side, c->ev_fork, 0)) != cudaSuccess) return e;
    k_ythomas_low<T><<<(nlow + 127) / 128, 128, 0, c->side>>>(make_geo<T>(c), c->m64full, c->yRM64, c->yCP64,
                                                              (CT*)c->spec, (double2*)c->ylow, c->KL, c->TSy, c->sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(c->ev_join, c->side)) != cudaSuccess) return e;
    k_ythomas<T, float, 16><<<gy, 128, 0, c->stream>>>(make_geo<T>(c), c->m64full, (const float*)c->yRM,
                                                       (const float*)c->yCP, (CT*)c->spec, c->KL, c->TSy, c->sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = cudaStreamWaitEvent(c->stream, c->ev_join, 0);
  }
  e = e != cudaSuccess ? e : cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (launch_zfft_r(c, 1, &e)) return e;
  k_zfft<T><<<gz, nthrz, smemz, c->stream>>>(make_geo<T>(c), (CT*)c->spec, c->planz, (const CT*)c->twz, TKX, 1, c->sc);
  return cudaGetLastError();
}
// Forward z transform of the spectrum alone (the first step of the spectral solve).
template <class T> static cudaError_t zfft_fwd_t(ch3d_ctx* c) {
  typedef typename CplxOf<T>::type CT;
  cudaError_t e;
  if (launch_zfft_r(c, 0, &e)) return e;
  const int nz = c->nz;
  int TKX = kFFTSmem / (2 * nz * (int)sizeof(CT));
  int t = 1;
  while (t * 2 <= TKX && t * 2 <= 16) t *= 2;
  TKX = t;
  static PerDevice attr;  // per precision (template instance)
  if ((e = smem_limit_once(attr, c->device, k_zfft<T>, 200 * 1024)) != cudaSuccess) return e;
  dim3 gz((c->nxh + TKX - 1) / TKX, c->ny);
  k_zfft<T><<<gz, 256, (size_t)2 * TKX * nz * sizeof(CT), c->stream>>>(make_geo<T>(c), (CT*)c->spec, c->planz,
                                                                      (const CT*)c->twz, TKX, 0, c->sc);
  return cudaGetLastError();
}
cudaError_t launch_zfft_forward(ch3d_ctx* c) { return c->fp32 ? zfft_fwd_t<float>(c) : zfft_fwd_t<double>(c); }

template <class T> static cudaError_t yfactors_t(ch3d_ctx* c) {
  const dim3 g((c->nxh + 127) / 128, c->nz / 2 + 1);
  if (y_periodic(c)) {  // periodic y (FP64 only)
    k_ycyclic_factors<<<g, 128, 0, c->stream>>>(c->m64full, c->wave, c->nx, c->ny, c->nxh, (double*)c->yRM,
                                                (double*)c->yCP, c->yA2);
  } else if (!c->fp32) {
    k_ythomas_factors<double><<<g, 128, 0, c->stream>>>(c->m64full, c->wave, c->nx, c->ny, (double*)c->yRM,
                                                        (double*)c->yCP, c->nxh, c->nxh);
  } else {
    k_ythomas_factors<float><<<g, 128, 0, c->stream>>>(c->m64full, c->wave, c->nx, c->ny, (float*)c->yRM,
                                                       (float*)c->yCP, c->nxh, c->nxh);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_ythomas_factors<double><<<dim3(1, c->KL + 1), 128, 0, c->stream>>>(c->m64full, c->wave, c->nx, c->ny, c->yRM64,
                                                                        c->yCP64, c->TSy,
                                                                        c->nxh < c->TSy ? c->nxh : c->TSy);
  }
  return cudaGetLastError();
}
cudaError_t launch_ysolve_factors(ch3d_ctx* c) { return c->fp32 ? yfactors_t<float>(c) : yfactors_t<double>(c); }

cudaError_t launch_poisson_spectral(ch3d_ctx* c) { return c->fp32 ? spectral_t<float>(c) : spectral_t<double>(c); }

template <class T> static cudaError_t xifft_t(ch3d_ctx* c) {
  typedef typename CplxOf<T>::type CT;
  cudaError_t e;
  if (launch_xifft_r(c, &e)) return e;  // register FFT when the length has a plan
  T** f = (T**)c->f;
  const int M = c->nx / 2;
  const int LPB = lines_per_block<T>(M);
  const int nlines = c->ny * c->nz;
  size_t smem = (size_t)2 * LPB * M * sizeof(CT);
  static PerDevice attr;  // per precision (template instance)
  if ((e = smem_limit_once(attr, c->device, k_xifft<T>, 200 * 1024)) != cudaSuccess) return e;
  const int nthr = 256;
  k_xifft<T><<<(nlines + LPB - 1) / LPB, nthr, smem, c->stream>>>(make_geo<T>(c), (const CT*)c->spec, f[10], c->planx,
                                                                 (const CT*)c->twx, (const CT*)c->twr, LPB,
                                                                 (T)c->normfft, c->sc);
  return cudaGetLastError();
}
cudaError_t launch_xifft(ch3d_ctx* c) { return c->fp32 ? xifft_t<float>(c) : xifft_t<double>(c); }

template <class T> static cudaError_t proj_t(ch3d_ctx* c, int mode) {
  if (c->march) return launch_proj_march(c, mode, false);
  T** f = (T**)c->f;
  T* in[3] = {mode == 1 ? f[0] : f[12], mode == 1 ? f[1] : f[13], mode == 1 ? f[2] : f[14]};
  k_proj<T><<<cell_grid(c), cell_block(), 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), in[0], in[1], in[2], f[0],
                                                          f[1], f[2], f[3], f[10], c->part, mode, c->sc, f[11]);
  return cudaGetLastError();
}
cudaError_t launch_proj(ch3d_ctx* c, int mode) { return c->fp32 ? proj_t<float>(c, mode) : proj_t<double>(c, mode); }
cudaError_t launch_proj_diag(ch3d_ctx* c) { return launch_proj_march(c, 0, true); }
cudaError_t launch_diag_reset(ch3d_ctx* c) {
  k_diag_reset<<<1, 1, 0, c->stream>>>(c->sc);
  return cudaGetLastError();
}

template <class T> static cudaError_t bulk_t(ch3d_ctx* c) {
  if (c->march) return launch_bulk_march(c);
  T** f = (T**)c->f;
  k_bulk_partial<T><<<cell_grid(c), cell_block(), 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], c->part);
  return cudaGetLastError();
}
cudaError_t launch_bulk_partials(ch3d_ctx* c) { return c->fp32 ? bulk_t<float>(c) : bulk_t<double>(c); }

// rows per k_diag block: whole columns when the x-z plane alone gives about
// eight blocks per SM, shorter chunks on small grids
static int diag_rows(const ch3d_ctx* c) {
  const long long cols = (long long)((c->nx + 31) / 32) * ((c->nz + 3) / 4);
  const long long chunks = (148LL * 8 + cols - 1) / cols;
  const int rows = (int)((c->ny + chunks - 1) / chunks);
  return rows < 8 ? 8 : rows;
}
static dim3 diag_grid(const ch3d_ctx* c) {
  const int rows = diag_rows(c);
  return dim3((c->nx + 31) / 32, (c->nz + 3) / 4, (c->ny + rows - 1) / rows);
}
int diag_npart(const ch3d_ctx* c) {
  const dim3 g = diag_grid(c);
  return (int)(g.x * g.y * g.z);
}

template <class T> static cudaError_t diag_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  k_diag_reset<<<1, 1, 0, c->stream>>>(c->sc);
  k_diag<T><<<diag_grid(c), 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], f[1], f[2], c->part2, c->sc,
                                                 diag_rows(c));
  return cudaGetLastError();
}
cudaError_t launch_diag(ch3d_ctx* c) { return c->fp32 ? diag_t<float>(c) : diag_t<double>(c); }

template <class T> static cudaError_t divmax_t(ch3d_ctx* c, unsigned long long* slot) {
  T** f = (T**)c->f;
  k_divmax<T><<<cell_grid(c), cell_block(), 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], f[1], f[2], slot);
  return cudaGetLastError();
}
template <class T> __global__ void k_fill_row0(T* __restrict__ a, int nx, int ny, int nz, T v) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nx * nz) return;
  const int i = (int)(t % nx), k = (int)(t / nx);
  a[i + (long long)nx * ny * k] = v;
}
// FP64 <-> FP32 conversion of n values (mixed-precision upload/download)
__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    b[t] = (float)a[t];
}
__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    b[t] = (double)a[t];
}
cudaError_t launch_convert(ch3d_ctx* c, const void* src, void* dst, long long n, int to_f32) {
  const long long nb = (n + 255) / 256;
  const unsigned g = (unsigned)(nb < 148LL * 32 ? nb : 148LL * 32);
  if (n <= 0) return cudaSuccess;
  if (to_f32) k_f64_to_f32<<<g, 256, 0, c->stream>>>((const double*)src, (float*)dst, n);
  else k_f32_to_f64<<<g, 256, 0, c->stream>>>((const float*)src, (double*)dst, n);
  return cudaGetLastError();
}

cudaError_t launch_fill_row0(ch3d_ctx* c, int q, double v) {
  const unsigned nb = (unsigned)(((long long)c->nx * c->nz + 255) / 256);
  if (c->fp32) k_fill_row0<float><<<nb, 256, 0, c->stream>>>((float*)c->f[q], c->nx, c->ny, c->nz, (float)v);
  else k_fill_row0<double><<<nb, 256, 0, c->stream>>>((double*)c->f[q], c->nx, c->ny, c->nz, v);
  return cudaGetLastError();
}

cudaError_t launch_divmax(ch3d_ctx* c, unsigned long long* slot) {
  return c->fp32 ? divmax_t<float>(c, slot) : divmax_t<double>(c, slot);
}

// ---------------------------------------------------------------------------
// clcStat_CH moment sums (src/CFD_2nd/m_FlowType_Channel.f90:175-330), FP64
// accumulation in both precision modes.  Block (j, k-chunk); blockIdx.x == ny
// is the nyp row (:296-316).  Partials are summed in a fixed order by
// k_stats_finalize, so the statistics are deterministic.
// ---------------------------------------------------------------------------
#define CH3D_NSTAT 35

template <class T>
__device__ __forceinline__ double fd(const T* a, const Geo<T>& g, int comp, int i, int j, int k) {
  return (double)fld(a, g, comp, i, j, k);
}

template <class T>
__global__ void __launch_bounds__(256) k_stats(Geo<T> g, Metrics<double> m, const T* __restrict__ ux,
                                               const T* __restrict__ uy, const T* __restrict__ uz,
                                               const T* __restrict__ pr, double* __restrict__ part, int kch) {
  __shared__ double wred[CH3D_NSTAT][8];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int j = blockIdx.x;  // 0..ny-1 interior rows (jc = j+1); ny: the nyp row
  const int k0 = blockIdx.y * kch, k1 = min(nz, k0 + kch);
  double S[CH3D_NSTAT];
#pragma unroll
  for (int q = 0; q < CH3D_NSTAT; ++q) S[q] = 0.0;
  const double rdx = (double)g.rdx, rdz = (double)g.rdz, rdx2 = (double)g.rdx2, rdz2 = (double)g.rdz2;
  const double rdxh = rdx * 0.5;
  if (j < ny) {
    const int jc = j + 1;
    const double InterpY1 = 0.5 * m.yinterp[jc], InterpY2 = 0.5 - InterpY1;
    const double cac = m.rdyc[jc], cacU = m.rdyc[jc + 1], caj = m.rdyp[jc];
    for (int k = k0; k < k1; ++k) {
      const int km = wrapm(k, nz), kp = wrapp(k, nz);
      for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int im = wrapm(i, nx), ip = wrapp(i, nx);
        const double uxloc = fd(ux, g, 0, i, j, k), uyloc = fd(uy, g, 1, i, j, k), uzloc = fd(uz, g, 2, i, j, k);
        const double prloc = fd(pr, g, 3, i, j, k);
        const double ux_ip = fd(ux, g, 0, ip, j, k), ux_im = fd(ux, g, 0, im, j, k);
        const double ux_jm = fd(ux, g, 0, i, j - 1, k), ux_jp = fd(ux, g, 0, i, j + 1, k);
        const double ux_km = fd(ux, g, 0, i, j, km), ux_kp = fd(ux, g, 0, i, j, kp);
        const double uy_jp = fd(uy, g, 1, i, j + 1, k), uy_im = fd(uy, g, 1, im, j, k), uy_ip = fd(uy, g, 1, ip, j, k);
        const double uy_jm = fd(uy, g, 1, i, j - 1, k), uy_km = fd(uy, g, 1, i, j, km), uy_kp = fd(uy, g, 1, i, j, kp);
        const double uy_im_jp = fd(uy, g, 1, im, j + 1, k);
        const double uz_kp = fd(uz, g, 2, i, j, kp), uz_km = fd(uz, g, 2, i, j, km);
        const double uz_im = fd(uz, g, 2, im, j, k), uz_ip = fd(uz, g, 2, ip, j, k);
        const double uz_jm = fd(uz, g, 2, i, j - 1, k), uz_jp = fd(uz, g, 2, i, j + 1, k);
        const double uxCell = 0.5 * (uxloc + ux_ip);
        const double uyCell = 0.5 * (uyloc + uy_jp);
        const double uzCell = 0.5 * (uzloc + uz_kp);
        const double prloc2 = InterpY1 * (fd(pr, g, 3, im, j - 1, k) + fd(pr, g, 3, i, j - 1, k)) +
                              InterpY2 * (fd(pr, g, 3, im, j, k) + prloc);
        const double dudx = (ux_ip - uxloc) * rdx, dudy = (uxloc - ux_jm) * cac, dudz = (uxloc - ux_km) * rdz;
        const double dvdx = (uyloc - uy_im) * rdx, dvdy = (uy_jp - uyloc) * caj, dvdz = (uyloc - uy_km) * rdz;
        const double dwdx = (uzloc - uz_im) * rdx, dwdy = (uzloc - uz_jm) * cac, dwdz = (uz_kp - uzloc) * rdz;
        const double dudxx = (ux_ip - 2.0 * uxloc + ux_im) * rdx2;
        const double dudyy = m.ap2c[jc] * ux_jp + m.ac2c[jc] * uxloc + m.am2c[jc] * ux_jm;
        const double dudzz = (ux_kp - 2.0 * uxloc + ux_km) * rdz2;
        const double dvdxx = (uy_ip - 2.0 * uyloc + uy_im) * rdx2;
        const double dvdyy = m.ap2p[jc] * uy_jp + m.ac2p[jc] * uyloc + m.am2p[jc] * uy_jm;
        const double dvdzz = (uy_kp - 2.0 * uyloc + uy_km) * rdz2;
        const double dwdxx = (uz_ip - 2.0 * uzloc + uz_im) * rdx2;
        const double dwdyy = m.ap2c[jc] * uz_jp + m.ac2c[jc] * uzloc + m.am2c[jc] * uz_jm;
        const double dwdzz = (uz_kp - 2.0 * uzloc + uz_km) * rdz2;
        const double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
        const double dudxC = (ux_ip - ux_im) * rdxh;
        const double dvdxU = (uy_jp - uy_im_jp) * rdx;
        const double dudyU = (ux_jp - uxloc) * cacU;
        const double dvdyM = (uy_im_jp - uy_im) * caj;
        const double dudzC = (InterpY1 * (fd(ux, g, 0, i, j - 1, kp) - fd(ux, g, 0, i, j - 1, km)) +
                              InterpY2 * (ux_kp - ux_km)) * rdz;
        const double dvdzC = (fd(uy, g, 1, im, j, kp) - fd(uy, g, 1, im, j, km) + uy_kp - uy_km) * rdz * 0.25;
        S[0] += uxloc; S[1] += uyloc; S[2] += uzloc; S[3] += prloc;
        S[4] += uxloc * uxloc; S[5] += uyloc * uyloc; S[6] += uzloc * uzloc; S[7] += prloc * prloc;
        S[8] += uxCell * uyCell; S[9] += uyCell * uzCell; S[10] += uxCell * uzCell;
        S[11] += uxCell * prloc; S[12] += uyCell * prloc; S[13] += uzCell * prloc;
        S[14] += uxCell * uxCell * uyCell; S[15] += uyloc * uyloc * uyloc; S[16] += uzCell * uzCell * uyCell;
        S[17] += uxCell * uyCell * uyCell; S[18] += uxloc * uxloc * uxloc; S[19] += uzloc * uzloc * uzloc;
        S[20] += uxloc * uxloc * uxloc * uxloc; S[21] += uyloc * uyloc * uyloc * uyloc;
        S[22] += uzloc * uzloc * uzloc * uzloc;
        S[23] += prloc * dudx; S[24] += prloc * dvdy; S[25] += prloc * dwdz;
        S[26] += prloc2 * (dudy + dvdx);
        S[27] += uxloc * (dudxx + dudyy + dudzz); S[28] += uyloc * (dvdxx + dvdyy + dvdzz);
        S[29] += uzloc * (dwdxx + dwdyy + dwdzz);
        S[30] += dudxC * (dvdxU + dvdx) * 0.5 + (dudyU + dudy) * (dvdyM + dvdy) * 0.25;
        S[31] += dudzC * dvdzC;
        S[32] += vor_x * vor_x; S[33] += vor_y * vor_y; S[34] += vor_z * vor_z;
      }
    }
  } else {
    // jc = nyp: ghost row above the last cell (SetBC_and_UpdateHalo values)
    const int jc = ny + 1, jm = ny - 1;
    const double cac = m.rdyc[jc];
    const double InterpY1 = 0.5 * m.yinterp[jc], InterpY2 = 0.5 - InterpY1;
    for (int k = k0; k < k1; ++k)
      for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int im = wrapm(i, nx);
        const double prloc2 = InterpY1 * (fd(pr, g, 3, im, jm, k) + fd(pr, g, 3, i, jm, k)) +
                              InterpY2 * (fd(pr, g, 3, im, ny, k) + fd(pr, g, 3, i, ny, k));
        const double dudy = (fd(ux, g, 0, i, ny, k) - fd(ux, g, 0, i, jm, k)) * cac;
        const double dwdy = (fd(uz, g, 2, i, ny, k) - fd(uz, g, 2, i, jm, k)) * cac;
        const double vor_x = dwdy, vor_z = -dudy;
        S[26] += prloc2 * (dudy + 0.0);
        S[32] += vor_x * vor_x;
        S[34] += vor_z * vor_z;
      }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < CH3D_NSTAT; ++q) {
    double v = S[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) wred[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < CH3D_NSTAT) {
    double v = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += wred[threadIdx.x][q];
    part[((size_t)j * gridDim.y + blockIdx.y) * CH3D_NSTAT + threadIdx.x] = v;
  }
}

// SumStat(:,jc) += sum of the partials * inxz (m_FlowType_Channel.f90:290-293);
// PrGradsum += PrGradAver (:318).
__global__ void k_stats_finalize(const double* __restrict__ part, int nch, double inxz, double* __restrict__ sumstat,
                                 DevScalars* sc, double* prgradsum) {
  const int j = blockIdx.x, q = threadIdx.x;
  if (q < CH3D_NSTAT) {
    double v = 0.0;
    for (int c = 0; c < nch; ++c) v += part[((size_t)j * nch + c) * CH3D_NSTAT + q];
    sumstat[(size_t)j * CH3D_NSTAT + q] += v * inxz;
  }
  if (j == 0 && q == 0) *prgradsum += sc->PrGradAver;
}

template <class T> static cudaError_t stats_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  const int kch = (c->nz + 7) / 8;
  const int nch = (c->nz + kch - 1) / kch;
  k_stats<T><<<dim3(c->ny + 1, nch), 256, 0, c->stream>>>(make_geo<T>(c), c->m64full, f[0], f[1], f[2], f[3],
                                                           c->statpart, kch);
  k_stats_finalize<<<c->ny + 1, 64, 0, c->stream>>>(c->statpart, nch, 1.0 / ((double)c->nx * (double)c->nz), c->stat,
                                                   c->sc, c->stat + (size_t)CH3D_NSTAT * (c->ny + 1));
  return cudaGetLastError();
}
cudaError_t launch_stats(ch3d_ctx* c) { return c->fp32 ? stats_t<float>(c) : stats_t<double>(c); }

// ---------------------------------------------------------------------------
// Allocation-free Poisson solve (ch3d_poisson_noalloc in include/ch3d.h).
// Its working memory is this file-scope device array, present on every GPU
// that loads the library until the process exits.  In host code the name
// g_noalloc_scratch is only a host-side stand-in for the symbol; the device
// address is obtained once per device with cudaGetSymbolAddress (with that
// device current) and cached.  All calls share the array.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[CH3D_NOALLOC_SCRATCH_BYTES];

namespace {
// per device: the scratch array's device address and the kernels' shared-memory limits set
PerDevice g_noalloc_site;
void* g_noalloc_addr[kMaxDevices] = {nullptr};
constexpr int kNoallocSmemLimit = 200 * 1024;

size_t align256(size_t b) { return (b + 255) / 256 * 256; }
}  // namespace

// Once per device (that device current): looks up the array's device address
// and sets the dynamic shared-memory limit of the four kernels the solve runs.
cudaError_t noalloc_scratch_address(int dev, void** out) {
  cudaError_t e = once_per_device(g_noalloc_site, dev, [&] {
    void* p = nullptr;
    cudaError_t r = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (r != cudaSuccess) return r;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((r = cudaFuncSetAttribute(k_prsrc_xfft<double>, a, kNoallocSmemLimit)) != cudaSuccess) return r;
    if ((r = cudaFuncSetAttribute(k_zfft<double>, a, kNoallocSmemLimit)) != cudaSuccess) return r;
    if ((r = cudaFuncSetAttribute(k_ysolve<double>, a, kNoallocSmemLimit)) != cudaSuccess) return r;
    if ((r = cudaFuncSetAttribute(k_xifft<double>, a, kNoallocSmemLimit)) != cudaSuccess) return r;
    g_noalloc_addr[dev] = p;
    return cudaSuccess;
  });
  if (e == cudaSuccess) *out = g_noalloc_addr[dev];
  return e;
}

// Launch shapes of the allocation-free solve: x-transform lines per block,
// z-transform kx lines per block, y-solve threads per system, and the dynamic
// shared memory of the x, z and y kernels.
struct NoallocShape {
  int LPB, TKX, P, TS;
  size_t smx, smz, smy;
};
static NoallocShape noalloc_shape(int nx, int ny, int nz) {
  NoallocShape s;
  const int M = nx / 2;
  s.LPB = lines_per_block<double>(M);
  int TKX = kFFTSmem / (2 * nz * (int)sizeof(double2));
  int tk = 1;
  while (tk * 2 <= TKX && tk * 2 <= 16) tk *= 2;
  s.TKX = tk;
  int P = 16;
  while (P > 1 && ny < 2 * P) P >>= 1;
  s.P = P;
  s.TS = 8;
  const int Q = P - 1;
  s.smx = (size_t)2 * s.LPB * M * sizeof(double2);
  s.smz = (size_t)2 * s.TKX * nz * sizeof(double2);
  s.smy = (size_t)ny * s.TS * (sizeof(double2) + 2 * sizeof(double)) +
          (size_t)s.TS * (Q > 0 ? Q : 1) * (2 * sizeof(double2) + 5 * sizeof(double)) + 16;
  return s;
}

// Largest dynamic shared memory (bytes) one kernel of the solve of an
// nx x ny x nz grid asks for; the solve runs only where it is within
// noalloc_smem_limit().
size_t noalloc_smem(int nx, int ny, int nz) {
  const NoallocShape s = noalloc_shape(nx, ny, nz);
  size_t m = s.smx > s.smz ? s.smx : s.smz;
  return m > s.smy ? m : s.smy;
}
size_t noalloc_smem_limit() { return (size_t)kNoallocSmemLimit; }

// Bytes of scratch the solve of an nx x ny x nz grid needs.
size_t noalloc_bytes(int nx, int ny, int nz) {
  const int nxh = nx / 2 + 1, M = nx / 2;
  size_t b = align256((size_t)nxh * ny * nz * sizeof(double2));
  b += align256((size_t)4 * (ny + 3) * sizeof(double));     // rdyp, am2Pr, ac2Pr, ap2Pr
  b += align256((size_t)(nx + nz) * sizeof(double));        // WaveNumX | WaveNumZ
  b += align256((size_t)(M + M + 1 + nz) * sizeof(double2)); // twiddles
  b += align256(sizeof(DevScalars));
  return b;
}

cudaError_t poisson_noalloc(int nx, int ny, int nz, double xlx, double zlz, const double* yp, int bclo, int bchi,
                            const double* d_src, double* d_phi, cudaStream_t st, const FFTPlanDev& planx,
                            const FFTPlanDev& planz) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  void* base = nullptr;
  e = noalloc_scratch_address(dev, &base);
  if (e != cudaSuccess) return e;
  const int nxh = nx / 2 + 1, M = nx / 2, L = ny + 3;
  unsigned char* p = (unsigned char*)base;
  double2* spec = (double2*)p;
  p += align256((size_t)nxh * ny * nz * sizeof(double2));
  double* met = (double*)p;
  p += align256((size_t)4 * L * sizeof(double));
  double* wave = (double*)p;
  p += align256((size_t)(nx + nz) * sizeof(double));
  double2* tw = (double2*)p;
  p += align256((size_t)(M + M + 1 + nz) * sizeof(double2));
  DevScalars* sc = (DevScalars*)p;

  // host tables: the Poisson metrics of InitMeshAndMetries (m_MeshAndMetries.f90:186-240),
  // the modified wavenumbers (m_Poisson.f90:38-66) and the FFT twiddles
  std::vector<double> h(4 * (size_t)L, 0.0), dyp(L, 0.0), dyc(L, 0.0), yc(L, 0.0), rdyc(L, 0.0);
  const int nyp = ny + 1;
  auto Y = [&](int j) { return yp[j - 1]; };
  for (int j = 1; j <= ny; ++j) { yc[j] = 0.5 * (Y(j) + Y(j + 1)); dyp[j] = Y(j + 1) - Y(j); }
  dyp[0] = dyp[1]; dyp[nyp] = dyp[ny];
  for (int j = 2; j <= ny; ++j) dyc[j] = yc[j] - yc[j - 1];
  dyc[1] = dyp[1]; dyc[nyp] = dyp[ny];
  double* rdyp = h.data();
  double *am = h.data() + L, *ac = h.data() + 2 * L, *ap = h.data() + 3 * L;
  for (int j = 0; j <= nyp; ++j) rdyp[j] = 1.0 / dyp[j];
  for (int j = 1; j <= nyp; ++j) rdyc[j] = 1.0 / dyc[j];
  for (int j = 1; j <= ny; ++j) { am[j] = rdyp[j] * rdyc[j]; ap[j] = rdyp[j] * rdyc[j + 1]; }
  if (bclo != 0) { am[1] = 0.0; ap[1] = rdyp[1] * rdyc[2]; }
  if (bchi != 0) { am[ny] = rdyp[ny] * rdyc[ny]; ap[ny] = 0.0; }
  for (int j = 1; j <= ny; ++j) ac[j] = -(am[j] + ap[j]);
  const double PIv = 3.141592653589793238462643383279502884;
  const double rdx = (double)nx / xlx, rdz = (double)nz / zlz;
  std::vector<double> w(nx + nz);
  for (int i = 0; i < nx; ++i) w[i] = 2.0 * rdx * rdx * (std::cos(2.0 * PIv * (double)i / (double)nx) - 1.0);
  for (int k = 0; k < nz; ++k) w[nx + k] = 2.0 * rdz * rdz * (std::cos(2.0 * PIv * (double)k / (double)nz) - 1.0);
  std::vector<double2> t(M + M + 1 + nz);
  auto fill = [&](double2* o, int n, int cnt) {
    for (int q = 0; q < cnt; ++q) {
      long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)q / (long double)n;
      o[q] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
  };
  fill(t.data(), M, M);
  fill(t.data() + M, nx, M + 1);
  fill(t.data() + 2 * M + 1, nz, nz);
  if ((e = cudaMemcpyAsync(met, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(wave, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(tw, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  // what must start at zero: the status word and the divergence maximum
  if ((e = cudaMemsetAsync(sc, 0, sizeof(DevScalars), st)) != cudaSuccess) return e;

  Geo<double> g;
  std::memset(&g, 0, sizeof(g));
  g.nx = nx; g.ny = ny; g.nz = nz; g.nxh = nxh; g.N = (long long)nx * ny * nz;
  g.rdx = rdx; g.rdz = rdz; g.rdx2 = rdx * rdx; g.rdz2 = rdz * rdz;
  g.bc.lo = bclo; g.bc.hi = bchi;
  g.bc.dyp1 = dyp[1]; g.bc.dypN = dyp[nyp];
  Metrics<double> m;
  std::memset(&m, 0, sizeof(m));
  m.rdyp = met; m.am2Pr = met + L; m.ac2Pr = met + 2 * L; m.ap2Pr = met + 3 * L;
  const double2* twx = tw;
  const double2* twr = tw + M;
  const double2* twz = tw + 2 * M + 1;

  // forward x transform of the source (mode 2: the source is read as is)
  const NoallocShape sh = noalloc_shape(nx, ny, nz);
  const int LPB = sh.LPB, TKX = sh.TKX, P = sh.P, TS = sh.TS;
  const int nlines = ny * nz;
  k_prsrc_xfft<double><<<(nlines + LPB - 1) / LPB, 256, sh.smx, st>>>(g, m, d_src, d_src, d_src, spec, planx, twx,
                                                                      twr, LPB, 2, sc, nullptr);
  dim3 gz((nxh + TKX - 1) / TKX, ny);
  k_zfft<double><<<gz, 256, sh.smz, st>>>(g, spec, planz, twz, TKX, 0, sc);
  k_ysolve<double><<<dim3((nxh + TS - 1) / TS, nz), TS * P < 64 ? 64 : TS * P, sh.smy, st>>>(g, m, wave, spec, TS, P,
                                                                                              sc);
  k_zfft<double><<<gz, 256, sh.smz, st>>>(g, spec, planz, twz, TKX, 1, sc);
  k_xifft<double><<<(nlines + LPB - 1) / LPB, 256, sh.smx, st>>>(g, spec, d_phi, planx, twx, twr, LPB,
                                                                 1.0 / ((double)nx * (double)nz), sc);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the host tables above are pageable and local to this call
  return cudaStreamSynchronize(st);
}

}  // namespace ch3d
