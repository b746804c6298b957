// ch3d_common.cuh -- shared device types for the B200 channel-flow step.
//
// Device layout (all fields): interior cells only, Fortran order with i
// fastest, 0-based index idx = i + nx*(j + ny*k), i in [0,nx), j in [0,ny),
// k in [0,nz); j = jc-1 of the reference.  Periodic x and z neighbours wrap;
// y ghost values are produced inline from the boundary rules of
// SetBC_and_UpdateHalo (src/CFD_2nd/m_BC_and_Halo.f90:232-344) instead of
// being stored, so no halo planes are kept or exchanged.
// Metric vectors keep the reference's Fortran index (jc = 0..nyp+1).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>

namespace ch3d {

// Devices a process may drive through this library (device ordinals 0..63).
constexpr int kMaxDevices = 64;

// One-time set-up at a launch site (function attributes, cached device
// properties) for each device a process drives; cudaFuncSetAttribute applies
// to the current device only, so each site keeps one flag per device.
struct PerDevice {
  std::atomic<unsigned long long> done{0ull};
};

inline std::recursive_mutex& setup_mutex() {
  static std::recursive_mutex m;
  return m;
}

// Runs setup() (returning cudaError_t) the first time `site` meets `device`,
// under a process-wide mutex; the device is marked only when setup succeeds,
// so a second host thread never launches before the attributes are in place
// and a failed set-up is retried on the next call.  The caller has `device`
// current.  Ordinals outside [0, kMaxDevices) give cudaErrorInvalidDevice.
template <class F> cudaError_t once_per_device(PerDevice& site, int device, F&& setup) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  const unsigned long long bit = 1ull << device;
  if (site.done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  std::lock_guard<std::recursive_mutex> lk(setup_mutex());
  if (site.done.load(std::memory_order_relaxed) & bit) return cudaSuccess;
  const cudaError_t e = setup();
  if (e == cudaSuccess) site.done.fetch_or(bit, std::memory_order_release);
  return e;
}

// SM count of a device, queried once (148, the B200's, if the query fails).
inline int sm_count(int device) {
  static PerDevice site;
  static int nsm[kMaxDevices] = {};
  const cudaError_t e = once_per_device(site, device, [&] {
    int v = 0;
    const cudaError_t r = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    if (r == cudaSuccess) nsm[device] = v;
    return r;
  });
  return e == cudaSuccess ? nsm[device] : 148;
}

// Shared-memory limit of one kernel, set once per device.
template <class K> cudaError_t smem_limit_once(PerDevice& site, int device, K kern, size_t bytes) {
  return once_per_device(site, device, [&] {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  });
}

template <class T> struct CplxOf;
template <> struct CplxOf<double> { typedef double2 type; };
template <> struct CplxOf<float> { typedef float2 type; };

__host__ __device__ inline double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ inline float2 mk(float a, float b) { return make_float2(a, b); }
template <class CT> __device__ __forceinline__ CT cadd(CT a, CT b) { return mk(a.x + b.x, a.y + b.y); }
template <class CT> __device__ __forceinline__ CT csub(CT a, CT b) { return mk(a.x - b.x, a.y - b.y); }
template <class CT> __device__ __forceinline__ CT cmul(CT a, CT b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class CT> __device__ __forceinline__ CT cconj(CT a) { return mk(a.x, -a.y); }

// Scalars that change during a run live on the device so that a whole time
// step can be replayed as one CUDA graph without host round trips.
struct DevScalars {
  double dt, SimTime;
  double pmGamma, pmTheta, pmAlpha, pmBeta, pmAlphaC, pmBetaT;
  double dpmdxns, PrGradNow, PrGradAver;
  double cflmp, uxm, s1tot1;
  double utau;                                          // LES: wall friction velocity of the step
  unsigned long long divmax1, divmax2, vmax[3], uddx;  // bit patterns of non-negative doubles
  int itime, status, ns, pad;
};

// Metric vectors (FP64 master copies; FP32 copies for the mixed path).
// Indexed with the reference's Fortran index.
template <class T> struct Metrics {
  const T* dyp;        // 0..nyp
  const T* rdyp;       // 0..nyp
  const T* rdyc;       // 0..nyp (1..nyp valid)
  const T* yinterp;    // YinterpCoe 1..nyp (0 unused)
  const T* ap2c; const T* ac2c; const T* am2c;    // 1..nyc
  const T* ap2p; const T* ac2p; const T* am2p;    // 1..nyc
  const T* ap2Pr; const T* ac2Pr; const T* am2Pr; // 1..nyc
  const T* s1coe;      // bulk-sum weight dyp(jc) or 0 (clcRhsX_PIMP :25-27), 1..nyc
};

// Boundary description for y (x and z are periodic).
struct YBc {
  int lo, hi;                     // BcOption(3), BcOption(4): -1 no-slip, -2 free-slip, 0 periodic
  double ux_lo, ux_hi, uz_lo, uz_hi, uy_lo, uy_hi;
  double dyp1, dypN;              // dyp(1), dyp(nyp)
};

template <class T> struct Geo {
  int nx, ny, nz, nxh;
  int order;                            // 2: src/CFD_2nd, 4: src/CFD_4th
  int implicit;                         // IsImplicit: 1 PIMP (CN in y), 2 FIMP (CN in x, y, z)
  int les;                              // LES_type > 0: variable viscosity nut
  long long N;
  T rdx, rdz, rdx2, rdz2;
  T ap1c, ac1c, am1c, ap3c, ac3c, am3c;  // constant for periodic x and z
  T xnu, g1, g2, g3;
  YBc bc;
};

__device__ __forceinline__ int wrapm(int i, int n) { return i == 0 ? n - 1 : i - 1; }
__device__ __forceinline__ int wrapp(int i, int n) { return i + 1 == n ? 0 : i + 1; }

// Field value with y ghost cells from the boundary rules
// (SetBC_and_UpdateHalo, src/CFD_2nd/m_BC_and_Halo.f90:241-282), or the
// periodic halo rows when y is periodic (BcOption(3:4) = 0).
// comp: 0 ux, 1 uy, 2 uz, 3 pressure.  j may be -1 .. ny.
template <class T>
__device__ __forceinline__ T fld(const T* __restrict__ a, const Geo<T>& g, int comp, int i, int j, int k) {
  const int nx = g.nx, ny = g.ny;
  if (j >= 0 && j < ny) return __ldg(a + i + (long long)nx * (j + (long long)ny * k));
  if (j < 0) {
    if (g.bc.lo == 0) return __ldg(a + i + (long long)nx * ((ny - 1) + (long long)ny * k));
    if (comp == 1) {  // uy(ic,0,kc) = uy_ym*2 - uy(ic,2,kc); never set (zero) in the 4th-order solver
      if (g.order == 4) return (T)0;
      return (T)(g.bc.uy_lo * 2.0) - __ldg(a + i + (long long)nx * (1 + (long long)ny * k));
    }
    T v = __ldg(a + i + (long long)nx * (0 + (long long)ny * k));
    if (comp == 3) return v;  // pressure(ic,0,kc) = pressure(ic,1,kc)
    double w = comp == 0 ? g.bc.ux_lo : g.bc.uz_lo;
    if (g.bc.lo == -1) return (T)(w * 2.0) - v;
    return v - (T)(w * g.bc.dyp1);
  }
  // j == ny  (reference index nyp)
  if (g.bc.hi == 0) return __ldg(a + i + (long long)nx * ((long long)ny * k));
  if (comp == 1) return (T)g.bc.uy_hi;  // uy(ic,nyp,kc) = uyBcValue(yp)
  T v = __ldg(a + i + (long long)nx * ((ny - 1) + (long long)ny * k));
  if (comp == 3) return v;
  double w = comp == 0 ? g.bc.ux_hi : g.bc.uz_hi;
  if (g.bc.hi == -1) return (T)(w * 2.0) - v;
  return (T)(w * g.bc.dypN) + v;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

}  // namespace ch3d
