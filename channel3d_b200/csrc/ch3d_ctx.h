// ch3d_ctx.h -- host-side context of the C ABI (no device code).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/ch3d.h"
#include "ch3d_common.cuh"
#include "fft.cuh"

#define CH3D_NRED 256

struct ch3d_ctx {
  ch3d_config cfg;
  int nx = 0, ny = 0, nz = 0, nxh = 0;
  long long N = 0, NS = 0;  // real points, complex spectral points
  bool fp32 = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // mixed path: a high-priority side stream for the FP64 low-mode Poisson y solves,
  // forked from and joined to `stream` around the FP32 solves
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  double last_ms = 0;

  // Runge-Kutta constants (src/CFD_2nd/m_Parameters.f90:291-306)
  int iadvance = 3;
  double gam[3] = {0, 0, 0}, the[3] = {0, 0, 0}, alp[3] = {0, 0, 0};

  // host metrics, Fortran-indexed (m_MeshAndMetries)
  double dx = 0, dz = 0, rdx = 0, rdz = 0, rdx2 = 0, rdz2 = 0, rdy2 = 0;
  double normfft = 1.0;
  std::vector<double> yp, yc, dyp, dyc, rdyp, rdyc, yinterp;
  std::vector<double> ap2c, ac2c, am2c, ap2p, ac2p, am2p, ap2Pr, ac2Pr, am2Pr;
  std::vector<double> am2cForCN, ap2cForCN, s1coe, WaveNumX, WaveNumZ;

  // device buffers
  void* f[15] = {nullptr};   // ux uy uz p hx hy hz rx ry rz phi nut u*x u*y u*z (precision T)
  void* ih[6] = {nullptr};   // 4th order: uxhx uyhx uzhx uxhz uyhz uzhz (precision T)
  double* hfac = nullptr;    // Helmholtz chunk/interface factors of the current substep
  void* mtab = nullptr;      // column-march row table of the current substep (precision T)
  double* pfac = nullptr;    // FIMP or periodic y: periodic x/z/y sweep factors of the current substep
  double* les_delta = nullptr;  // LES: DeltaCell (ny+2) | wall distance of the cell centres (ny+2)
  // learned closure (LES_type CH3D_LES_MLP)
  float* mlp_params = nullptr;   // CH3D_MLP_NPARAM FP32
  unsigned char* mlp_packed = nullptr;  // their BF16 operand image (k_mlp_pack)
  float mlp_norm[CH3D_SGS_NORM_FLOATS] = {0};
  bool mlp_ready = false;
  int* mlp_status = nullptr;
  double* sgs_tau = nullptr;     // 6 N stresses at the cell centres
  double* sgs_f = nullptr;       // 3 N stress-divergence forces at the velocity points
  void* yRM = nullptr;       // Poisson y-solve Thomas factors per mode (fixed for the run);
  void* yCP = nullptr;       // FP64, or FP32 in the mixed path
  double* yRM64 = nullptr;   // mixed path: FP64 factors of the low modes (kx < TSy, |kz| <= KL)
  double* yCP64 = nullptr;
  double* ylow = nullptr;    // mixed path: FP64 forward-sweep scratch of the low modes
  double* yA2 = nullptr;     // periodic y: the Poisson cyclic solve's closure vector per mode
  bool gsub = false;         // the march stops at g; divergence and projection substitute u*
  int KL = 8;
  int TSy = 8;               // kx extent of the FP64 low modes
  int Pv = 32;               // chunks of the partitioned velocity Helmholtz solves
  void* spec = nullptr;      // complex spectrum (kx,j,kz)
  void* met = nullptr;       // packed metric vectors (precision T)
  double* met64 = nullptr;   // FP64 copy (always)
  double* wave = nullptr;    // WaveNumX (nx) | WaveNumZ (nz), FP64
  void* twx = nullptr;       // W_{nx/2} table
  void* twr = nullptr;       // W_{nx} table, 0..nx/2
  void* twz = nullptr;       // W_{nz} table
  ch3d::DevScalars* sc = nullptr;
  double* part = nullptr;    // block partial sums of ux*s1coe (bulk constraint)
  double* part2 = nullptr;   // block partial sums of ux*dyp (CalcUxAver)
  double* red1 = nullptr;    // CH3D_NRED second-level sums of part
  double* red2 = nullptr;    // CH3D_NRED second-level sums of part2
  int npart = 0;
  bool march = false;        // 2nd-order PIMP without LES: march kernels, npart_m partial sums in part
  int npart_m = 0;
  void* spec2 = nullptr;     // second half spectrum of the 1-D spectra (allocated at their first sample)
  double* specacc = nullptr; // EnergySpecX (nxh, ny, 18) | EnergySpecZ (nz/2+1, ny, 18) sums (FP64)
  int nspectime = 0;
  double* stat = nullptr;    // SumStat(35, nyp) | PrGradsum [| SumGrad(98, nyp), 4th order] (FP64)
  double* statpart = nullptr;
  int nfstime = 0;
  double prgradsum = 0;
  long long bytes = 0;

  ch3d::FFTPlanDev planx, planz;
  ch3d::Metrics<double> m64;
  ch3d::Metrics<double> m64full;  // FP64 metrics (always the FP64 copy)
  ch3d::Metrics<float> m32;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  bool scalars_ready = false;
};

namespace ch3d {

// y periodic (BcOption(3:4) = 0): the triply periodic steps (FIMP_000, PIMP_0)
inline bool y_periodic(const ch3d_ctx* c) { return c->cfg.BcOption[2] == 0; }
// launchers (ch3d_step.cu)
cudaError_t launch_substep_setup(ch3d_ctx* c, int ns);
cudaError_t launch_step_begin(ch3d_ctx* c);
cudaError_t launch_step_end(ch3d_ctx* c);
cudaError_t launch_rhs(ch3d_ctx* c);
cudaError_t launch_uhat(ch3d_ctx* c);                  // stage path: Rhs arrays -> u*
// 2nd-order PIMP step: RHS + y solves as a column march (ch3d_march.cu)
cudaError_t launch_rhs_march(ch3d_ctx* c);             // u -> u*, Hist, with its row table
size_t march_table_bytes(int ny);
cudaError_t march_table_reset(ch3d_ctx* c);           // forget the cached factors
cudaError_t launch_proj_march(ch3d_ctx* c, int mode, bool diag);  // projection + pressure update + bulk partials
bool march_twisted(const ch3d_ctx* c);                 // the march runs as two-group (twisted) blocks
cudaError_t launch_div_bsub(ch3d_ctx* c);               // div(u*) from g into phi's array (gsub)
cudaError_t launch_proj_bsub(ch3d_ctx* c, bool diag);   // projection + pressure update from g (gsub)
bool xplan_exists(int m);                               // the register x FFT has a plan for m = nx/2
bool march_diag_fusable(const ch3d_ctx* c);            // the step diagnostics can ride on the last projection
cudaError_t launch_bulk_march(ch3d_ctx* c);            // bulk partials of an uploaded field
int march_npart(const ch3d_ctx* c);
cudaError_t launch_helm_factors(ch3d_ctx* c);
cudaError_t launch_prsrc_xfft(ch3d_ctx* c, int mode);  // mode 0: div(u*)/pmAlpha, 1: div(u), 2: source in phi,
                                                       // 3: div(u*) in phi's array, /pmAlpha (register FFT only)
cudaError_t launch_poisson_spectral(ch3d_ctx* c);      // z fwd, y solve, z inv
cudaError_t launch_xifft(ch3d_ctx* c);
// register-resident FFT kernels for the lengths with a plan (ch3d_rfft.cu);
// false: no plan, nothing launched
bool launch_prsrc_xfft_r(ch3d_ctx* c, int mode, cudaError_t* err);
bool launch_zfft_r(ch3d_ctx* c, int inverse, cudaError_t* err);
bool launch_xifft_r(ch3d_ctx* c, cudaError_t* err);
cudaError_t launch_ysolve_factors(ch3d_ctx* c);
cudaError_t launch_interp_state(ch3d_ctx* dst, const ch3d_ctx* src);  // Interp_uvwp onto dst's grid
cudaError_t launch_zfft_forward(ch3d_ctx* c);          // forward z transform of the spectrum alone
cudaError_t launch_spectra(ch3d_ctx* c, int jfor1, int jfor2);  // one sample of the 4th-order 1-D spectra
// allocation-free Poisson solve (static device scratch, ch3d_step.cu)
size_t noalloc_bytes(int nx, int ny, int nz);
size_t noalloc_smem(int nx, int ny, int nz);
size_t noalloc_smem_limit();
cudaError_t noalloc_scratch_address(int dev, void** out);
cudaError_t poisson_noalloc(int nx, int ny, int nz, double xlx, double zlz, const double* yp, int bclo, int bchi,
                            const double* d_src, double* d_phi, cudaStream_t st, const FFTPlanDev& planx,
                            const FFTPlanDev& planz);
cudaError_t launch_proj(ch3d_ctx* c, int mode);        // mode 0: u = u* - a grad phi, p update; 1: u -= grad phi
cudaError_t launch_proj_diag(ch3d_ctx* c);             // last substep: projection + step diagnostics (march path)
cudaError_t launch_diag_reset(ch3d_ctx* c);
cudaError_t launch_bulk_partials(ch3d_ctx* c);
cudaError_t launch_diag(ch3d_ctx* c);
int diag_npart(const ch3d_ctx* c);                     // partial sums k_diag writes to part2
cudaError_t launch_stats(ch3d_ctx* c);
cudaError_t launch_stats4(ch3d_ctx* c);
cudaError_t launch_divmax(ch3d_ctx* c, unsigned long long* slot);
cudaError_t launch_fill_row0(ch3d_ctx* c, int q, double v);  // field q: every j = 0 value := v
cudaError_t launch_convert(ch3d_ctx* c, const void* src, void* dst, long long n, int to_f32);  // FP64 <-> FP32
// 4th-order solver (ch3d_step4.cu)
cudaError_t launch_rhs4(ch3d_ctx* c);                  // stage path: interpolation + RhsX/Y/Z
cudaError_t launch_visc4_partials(ch3d_ctx* c);        // mean viscous stress partial sums -> part
int visc4_npart(const ch3d_ctx* c);                   // their count
cudaError_t launch_dissipation(ch3d_ctx* c, int* npart);  // CalcDissipationRate partials -> part2
cudaError_t launch_reduce_partials(ch3d_ctx* c, const double* in, int n, double* out);  // CH3D_NRED sums
// fully implicit and explicit 2nd-order steps (ch3d_step.cu, ch3d_fimp.cu)
cudaError_t launch_rhs_fimp(ch3d_ctx* c);              // clcRhsX/Y/Z_FIMP (or _FEXP) -> RhsX/Y/Z
cudaError_t launch_uhat_fexp(ch3d_ctx* c);             // clcU1/2/3Hat_FEXP: u* = u + RhsX/Y/Z
cudaError_t launch_ptri_xz(ch3d_ctx* c);               // periodic x and z sweeps of RhsX/Y/Z, in place
cudaError_t launch_ptri_y(ch3d_ctx* c);                // periodic y sweep (y periodic, FIMP or PIMP): u* = u + solution
size_t ptri_factor_doubles(int nx, int ny, int nz);
// LES (ch3d_les.cu), FP64
cudaError_t launch_mlp_pack(ch3d_ctx* c);              // parameter image of the closure's network
cudaError_t launch_fill_nut(ch3d_ctx* c);              // nut = xnu (learned closure)
cudaError_t launch_sgs_nut(ch3d_ctx* c);               // Clc_SGS_Vis -> nut
cudaError_t launch_rhs_les(ch3d_ctx* c);               // clcRhsX/Y/Z_PIMP_LES -> RhsX/Y/Z
cudaError_t launch_uhat_les(ch3d_ctx* c);              // clcU1/2/3Hat_PIMP_LES -> u*
cudaError_t launch_sgs_samples(ch3d_ctx* c, int fx, int fy, int fz, float* X, float* T);
}  // namespace ch3d
