/*
 * ch3d.h -- C ABI of the B200 implementation of Channel3d's RK3 time step.
 *
 * The Fortran host of the reference keeps its .prm input, its module call
 * sites and its restart/statistics layout, and binds these entry points
 * through ISO_C_BINDING.  Every function returns an int
 * status (CH3D_OK = 0); the message of the last failure of a thread is
 * available from ch3d_last_error().  Arrays crossing this boundary are plain
 * host pointers to real(8) data in Fortran (column-major) order.
 *
 * Array layouts (argument `layout`):
 *   CH3D_LAYOUT_INTERIOR   (1:nxc,1:nyc,1:nzc), the restart-file layout of
 *                          write_restart/read_restart
 *                          (src/CFD_2nd/m_IOAndVisu.f90:352-558).
 *   CH3D_LAYOUT_GHOST2     (0:nxc+2,0:nyc+2,0:nzc+2), the `mb1` bounds of the
 *                          2nd-order solver (src/CFD_2nd/m_Variables.f90:59-61).
 *   CH3D_LAYOUT_GHOST4     (-1:nxc+2,0:nyc+1,-1:nzc+2), the `mb1` bounds of the
 *                          4th-order solver (src/CFD_4th/m_Variables.f90:47-49).
 * Upload reads the interior of a ghosted array.  On download, ghost cells
 * are filled by the boundary rules and periodic halo copies of
 * SetBC_and_UpdateHalo / SetBC_and_UpdateHalo_pr with each tree's halo
 * widths (src/CFD_2nd/m_BC_and_Halo.f90:20-29,232-344,410-456;
 * src/CFD_4th/m_BC_and_Halo.f90:24-46,51-96,136-150); cells those routines
 * never write keep the values the host array had.
 *
 * Threading: one context = one CUDA stream on one device; a context is not
 * thread-safe, distinct contexts are independent.  Device memory is owned by
 * the context; host arrays are only borrowed during the call.
 */
#ifndef CH3D_H_
#define CH3D_H_

#if defined(__GNUC__)
#define CH3D_API __attribute__((visibility("default")))
#else
#define CH3D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CH3D_OK 0
#define CH3D_ERR_INVALID 1      /* bad argument or configuration */
#define CH3D_ERR_UNSUPPORTED 2  /* valid for the reference, not built here */
#define CH3D_ERR_CUDA 3         /* CUDA runtime failure */
#define CH3D_ERR_DIVERGED 4     /* div_limit or vel_limit exceeded (the
                                   reference's ErrT_Abort in ChannelIterate,
                                   src/CFD_2nd/m_ChannelSystem.f90:127-130) */
#define CH3D_ERR_NOMEM 5

#define CH3D_LAYOUT_INTERIOR 0
#define CH3D_LAYOUT_GHOST2 1
#define CH3D_LAYOUT_GHOST4 2

#define CH3D_PREC_FP64 0
#define CH3D_PREC_MIXED 1       /* FP32 fields, FP64 low-mode Poisson, bulk
                                   constraint and statistics; LES: the eddy
                                   viscosity, the closure's inputs and the
                                   variable-viscosity solves in FP64
                                   arithmetic on the FP32 fields */

/* LES closures; the reference's LES_type values (src/CFD_2nd/m_Parameters.f90:256-259)
   plus the closures added on top (no counterpart in the reference). */
#define CH3D_LES_NONE 0
#define CH3D_LES_WALE 2
#define CH3D_LES_MTS 3
#define CH3D_LES_SMAG_VD 10     /* Smagorinsky + van Driest damping */
#define CH3D_LES_MLP 11         /* learned closure, Smagorinsky fallback */
/* standardisation of the learned closure: in_mean[10], in_std[10],
   in_lo[10], in_hi[10] (training range of the standardised inputs),
   out_mean[6], out_std[6] */
#define CH3D_SGS_NORM_FLOATS 52

/* Configuration: the namelist variables of &BasicParam, &ubulk_Param and
   &LesOptions (src/CFD_2nd/m_Parameters.f90:273-277,
   src/CFD_2nd/m_TScheme.f90:47) that the time step reads, plus the
   precision mode. */
typedef struct ch3d_config {
  int order;              /* 2: src/CFD_2nd, 4: src/CFD_4th */
  int nxc, nyc, nzc;
  double xlx, yly, zlz;
  double xnu;
  double dtMax;
  int iCFL;               /* 1: dt from CFLc, 2: dt = dtMax */
  double CFLc;
  int ischeme;            /* 1 AB2, 2 RK2, 3 RK3 */
  int IsImplicit;         /* 1 PIMP (y Crank-Nicolson), 2 FIMP (x,z,y ADI) */
  int FlowType;           /* 1 channel, 2 half channel, 3 Taylor-Green vortex */
  int BcOption[6];        /* x-,x+,y-,y+,z-,z+ : 0 periodic, -1 no-slip, -2 free-slip;
                             x and z periodic; y periodic on both sides only with
                             IsImplicit = 2 in FP64 (clcU*Hat_FIMP_000,
                             src/CFD_2nd/m_TScheme.f90:151-157) */
  double uxBcValue[6], uyBcValue[6], uzBcValue[6];
  double gravity[3];
  int IsUxConst;
  double ubulk, ybulk1, ybulk2;
  int LES_type;
  int FilterType;
  double Cs;              /* Smagorinsky constant for CH3D_LES_SMAG_VD */
  double vel_limit, div_limit;
  int precision;          /* CH3D_PREC_* */
  int device;             /* CUDA device ordinal */
} ch3d_config;

/* Per-step diagnostics: what ChannelIterate logs
   (src/CFD_2nd/m_ChannelSystem.f90:138-153). */
typedef struct ch3d_step_info {
  double SimTime, dt, cflmp, divmax1, divmax2, vmax[3], uxm, PrGradAver;
  int itime;
  int status;             /* 0, or 1 div_limit / 2 vel_limit tripped */
} ch3d_step_info;

typedef struct ch3d_ctx ch3d_ctx;

/* Version string of the library. */
CH3D_API const char* ch3d_version(void);

/* Message of the last failed call on this thread (never NULL). */
CH3D_API const char* ch3d_last_error(void);

/* y grid of one mesh section, as clcCoord computes it
   (src/CFD_2nd/m_MeshAndMetries.f90:292-360): fills coordinate[id1..id2]
   (1-based Fortran indices into yp). */
CH3D_API int ch3d_mesh_section(double* yp, int id1, int id2, double c1, double c2,
                      int StretType, double cStret, int StretOption);

/* Whole y grid yp(1:nyp) from &MeshSection/&MeshOptions
   (src/CFD_2nd/m_MeshAndMetries.f90:122-160). */
CH3D_API int ch3d_mesh_y(int nyc, double yly, int nSection, const double* SectionLength,
                const int* nycSection, const int* StretType,
                const int* StretOption, const double* SectioncStret,
                double* yp);

/* Replaces InitMeshAndMetries + AllocateVariables + InitPoissonSolver +
   InitTimeScheme (src/CFD_2nd/m_ChannelSystem.f90:39-45): builds the metric
   vectors from yp(1:nyp) exactly as InitMeshAndMetries does
   (src/CFD_2nd/m_MeshAndMetries.f90:171-286) and allocates the device state. */
CH3D_API int ch3d_create(const ch3d_config* cfg, const double* yp, ch3d_ctx** out);

/* Frees the device state. */
CH3D_API int ch3d_destroy(ch3d_ctx* ctx);

/* Replaces read_restart + the ghost rebuild of ChannelInitialize
   (src/CFD_2nd/m_ChannelSystem.f90:54-63).  hist (3 arrays, interior layout,
   HistX|HistY|HistZ) may be NULL (zeros, as RK3 restarts use). */
CH3D_API int ch3d_upload_state(ch3d_ctx* ctx, int layout, const double* ux,
                      const double* uy, const double* uz, const double* p,
                      const double* hist);

/* Copies the state back to host arrays (write_restart's data). Any pointer may be NULL. */
CH3D_API int ch3d_download_state(ch3d_ctx* ctx, int layout, double* ux, double* uy,
                        double* uz, double* p, double* hist);

/* Replaces `nsteps` calls of ChannelIterate (src/CFD_2nd/m_ChannelSystem.f90:73-154;
   src/CFD_4th/m_ChannelSystem.f90:83-190) without statistics/IO.
   Returns CH3D_ERR_DIVERGED if a limit tripped (info->itime tells when). */
CH3D_API int ch3d_step(ch3d_ctx* ctx, int nsteps, ch3d_step_info* info);

/* Stage-level entry points, one per procedure pointer of the reference's
   substep (src/CFD_2nd/m_ChannelSystem.f90:91-124), for parity tests and for
   hosts that keep their own loop:
     0 PMcoeUpdate(ns) + Update_uy_ym   (m_Parameters.f90:329-342)
     1 clcRhsX/Y/Z                      (m_TSchemePIMP_inc.f90:7-325)
     2 clcU1Hat/U2Hat/U3Hat             (m_TSchemePIMP_inc.f90:392-740)
     3 clcPrSrc                         (m_TScheme.f90:213-241)
     4 clcPPE                           (m_Poisson.f90:1078-1201)
     5 FluidVelUpdate                   (m_TScheme.f90:281-306)
     6 PressureUpdate                   (m_TSchemePIMP_inc.f90:852-873)  */
CH3D_API int ch3d_stage(ch3d_ctx* ctx, int stage, int ns);

/* Internal arrays for inspection, interior layout: 0 ux, 1 uy, 2 uz,
   3 pressure, 4 HistXOld, 5 HistYOld, 6 HistZOld, 7 RhsX, 8 RhsY,
   9 prphi (the pressure correction of the last clcPPE), 10 nut (LES: the
   total viscosity of Clc_SGS_Vis, xnu included), 11 RhsZ, 12..14 the
   velocity after the Helmholtz solves (u*), 15..20 (CH3D_LES_MLP, read
   only) the SGS stresses tau_11 tau_12 tau_13 tau_22 tau_23 tau_33 at the
   cell centres of the last ch3d_sgs_viscosity or step. */
CH3D_API int ch3d_get_array(ch3d_ctx* ctx, int which, double* host);
CH3D_API int ch3d_set_array(ch3d_ctx* ctx, int which, const double* host);

/* Standalone pressure Poisson solve of clcPPE (src/CFD_2nd/m_Poisson.f90:1078-1201),
   src and phi in the interior layout. */
CH3D_API int ch3d_poisson(ch3d_ctx* ctx, const double* src, double* phi);

/* Projects the current velocity onto the discrete divergence-free space
   (Poisson solve of div(u) + FluidVelUpdate with pmAlpha = 1). */
CH3D_API int ch3d_project(ch3d_ctx* ctx, double* divmax_before, double* divmax_after);

/* Sets dt (iCFL = 2 runs only use dtMax). */
CH3D_API int ch3d_set_dt(ch3d_ctx* ctx, double dt);

/* Statistics: the moment sums of clcStat_CH (2nd order,
   src/CFD_2nd/m_FlowType_Channel.f90:175-330) or clcStat (4th order,
   src/CFD_4th/m_FlowCase.f90:330-640), accumulated on the device in FP64;
   fetch returns SumStat(35,nyp) in Fortran order, nfstime and PrGradsum,
   and optionally resets them (the gradient moments of the 4th order too). */
CH3D_API int ch3d_stats_accumulate(ch3d_ctx* ctx);
CH3D_API int ch3d_stats_fetch(ch3d_ctx* ctx, double* sumstat, int* nfstime,
                     double* prgradsum, int reset);

/* 4th order: one sample of the spectra of clcStat (src/CFD_4th/m_FlowCase.f90:
   642-935) from the current state, accumulated on the device in FP64.  1-D
   (clcSpectra1D): per row jc, in x (nxc/2+1 wavenumbers) and in z (nzc/2+1),
   18 spectra in the order of the iSpec1D* indices (:43-60): UU VV WW PP UV
   UV2, then for UU, VV, WW, PP the linear coherence spectra R1 I1 R2 against
   rows jForLCS(1) and jForLCS(2) (1..nyc/2, mirrored above the centre).  2-D
   (clcSpectra2D): per (kx, jc <= nyc/2, kz) the 9 spectra of the iSpec2D*
   indices (:62-72): UU VV WW PP UV and the coherence spectra R of UU, VV,
   WW, PP against row jForLCS(1), the two halves of the channel folded
   together.  The first call allocates a second half spectrum and the sums. */
CH3D_API int ch3d_spectra_accumulate(ch3d_ctx* ctx, int jForLCS1, int jForLCS2);

/* The sums EnergySpecX(nxc/2+1, nyc, 18), EnergySpecZ(nzc/2+1, nyc, 18) and
   EnergySpec2D(nxc/2+1, nyc/2, nzc/2+1, 9) in Fortran order (the SpecX /
   SpecZ files hold the 1-D sums divided by nSpectime; Spec2D the 2-D sums
   divided by nSpectime and weighted by Ratio2D, :1050-1100), and nSpectime;
   any pointer may be NULL; reset zeroes them. */
CH3D_API int ch3d_spectra_fetch(ch3d_ctx* ctx, double* specx, double* specz, double* spec2d, int* nSpectime,
                                int reset);

/* 4th order: the gradient moments SumGrad(98,nyp) of clcStat
   (HighOrderGradStat, src/CFD_4th/m_FlowCase.f90:485-589, the vGrad file's
   sums), Fortran order.  Fetch them before a resetting ch3d_stats_fetch. */
CH3D_API int ch3d_stats_fetch_grad(ch3d_ctx* ctx, double* sumgrad);

/* The Taylor-Green vortex statistic of the 2nd-order solver: clcStat_TG
   (src/CFD_2nd/m_FlowType_TGVortex.f90:87-113), *eps = xnu times the mean
   over the cells of CalcDissipationRate (src/CFD_2nd/m_Tools.f90:497-540,
   2 S_ij S_ij with the reference's stencils), of the current velocity: the
   value the reference writes to TG_dissp beside SimTime.  Synchronous;
   CH3D_ERR_UNSUPPORTED for a 4th-order context. */
CH3D_API int ch3d_dissipation(ch3d_ctx* ctx, double* eps);

/* LES: computes nut from the current velocity as the step does once per
   step, Clc_SGS_Vis (src/CFD_2nd/m_LESModels.f90:47-62) followed by the wall
   and periodic ghost rules of SetBC_and_UpdateHalo_SGS (:375-428).
   CH3D_LES_WALE and CH3D_LES_MTS follow Clc_SGS_WALE / Clc_SGS_MTS;
   CH3D_LES_SMAG_VD (no counterpart in the reference, whose Smagorinsky
   branch is empty) is nut = xnu + (Cs D Delta)^2 |S| with the van Driest
   damping D = 1 - exp(-y+/26), y+ from the x-z mean wall shear of the first
   cells. */
CH3D_API int ch3d_sgs_viscosity(ch3d_ctx* ctx);

/* Learned closure (LES_type = CH3D_LES_MLP; no counterpart in the
   reference): sets the network parameters (host FP32 array, CH3D_MLP_NPARAM
   values in the layout of include/ch3d_mlp.h) and the standardisation (host,
   CH3D_SGS_NORM_FLOATS values).  Network inputs per cell centre: the nine
   velocity gradients du_i/dx_j in wall units (g xnu / u_tau^2, order dudx
   dudy dudz dvdx dvdy dvdz dwdx dwdy dwdz) and y+; outputs: tau_11 tau_12
   tau_13 tau_22 tau_23 tau_33 / u_tau^2.  Points whose standardised input
   leaves [in_lo, in_hi] use the Smagorinsky / van Driest stress -2 nu_t S_ij.
   Must be called before the first step. */
CH3D_API int ch3d_sgs_mlp_set(ch3d_ctx* ctx, const float* params, const float* norm);

/* Training samples of the learned closure from the current (DNS) field:
   box filter over non-overlapping boxes of fx x fy x fz cells (volume
   weighted in y); per box the nine filtered velocity gradients in wall units
   and y+ (X, DEVICE, nbox x 10 FP32) and the subgrid stresses
   tau_ij = <u_i u_j> - <u_i><u_j> of the cell-centre velocities divided by
   u_tau^2 (T, DEVICE, nbox x 6 FP32), nbox = (nxc/fx) (nyc/fy) (nzc/fz).
   *nbox receives the count; X and T must hold that many rows. */
CH3D_API int ch3d_sgs_training_samples(ch3d_ctx* ctx, int fx, int fy, int fz, float* X, float* T, long long* nbox);

/* Device bytes held by the context. */
CH3D_API int ch3d_memory_bytes(ch3d_ctx* ctx, long long* bytes);

/* Runs `nsteps` steps launching kernel groups one by one, with CUDA events
   between them on the context's stream, and returns in out[0..5] the mean time
   (ms) per substep of each group: 0 RHS stencils, 1 y Helmholtz solves,
   2 divergence + forward x FFT, 3 z FFT + y Poisson solve + inverse z FFT,
   4 inverse x FFT, 5 projection + pressure update; out[6] is the time per step
   of the scalar and reduction kernels (CFL, substep coefficients,
   diagnostics).  The steps advance the state like ch3d_step. */
CH3D_API int ch3d_kernel_times(ch3d_ctx* ctx, int nsteps, double* out, int nout);

/* Allocation-free pressure Poisson solve: the solve of ch3d_poisson
   (periodic x and z, walls in y) for callers that cannot allocate device
   memory themselves, such as a host whose device memory is owned and fully
   reserved by another runtime, or a process in which every device allocation
   must go through the host application's own allocator.  It needs no context:
   the caller passes the grid (yp = yp(1:nyc+1)), the y boundary types
   (BcOption(3), BcOption(4): -1 no-slip, -2 free-slip) and DEVICE pointers to
   src and phi (nxc*nyc*nzc doubles each, interior layout), and `stream`
   (a cudaStream_t, or NULL for the legacy default stream) on the current
   device.  The call makes no device allocation of its own: its working memory
   is one file-scope device array of CH3D_NOALLOC_SCRATCH_BYTES in the library,
   which every GPU that loads the library holds until the process exits.  Grids
   whose spectrum and tables do not fit in it are rejected with
   CH3D_ERR_INVALID.  The first call on a device looks up the array's device
   address (cudaGetSymbolAddress) with that device current; make that first
   call before any stream capture.  All calls share the array and each call
   overwrites it, so calls whose work overlaps on the GPU (other streams,
   other host threads) race; serialise them.  The call returns after its work
   on `stream` has completed.  It has no counterpart in the reference. */
#define CH3D_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
CH3D_API int ch3d_poisson_noalloc(int nxc, int nyc, int nzc, double xlx, double zlz,
                                  const double* yp, int bc_ym, int bc_yp,
                                  const double* d_src, double* d_phi, void* stream);

/* Resamples the state of `src` onto the grid of `dst` and makes it dst's
   state, as the reference's interpolateField tool does between restart files
   (Interp_init / Interp_uvwp, Tool/interpolateField/src/m_Interp.f90:20-361):
   ux, uy, uz and p interpolated trilinearly at their own staggered positions
   of the new grid from the old field and its ghost cells
   (Tool/interpolateField/src/m_BC_and_Halo.f90:21-340), x and z in
   coordinates normalised by the domain lengths, y physical (the two grids
   share yly); ux rescaled to dst's ubulk when dst holds the flow rate
   (IsUxConst, :225-236).  dst's Hist is zero afterwards (an RK3 restart).
   Both contexts on one device, same precision. */
CH3D_API int ch3d_interp_state(ch3d_ctx* dst, const ch3d_ctx* src);

/* Time of the last ch3d_step call's kernels, measured with CUDA events on the
   context's stream (milliseconds). */
CH3D_API int ch3d_last_step_ms(ch3d_ctx* ctx, double* ms);

/* Kernel layout the context chose for its step (no counterpart in the
   reference; for profiling and benchmark labels): *flags receives the OR of */
#define CH3D_PATH_MARCH 1    /* RHS and y Helmholtz solves as one column march */
#define CH3D_PATH_TWISTED 2  /* the march runs from both walls (few column tiles) */
#define CH3D_PATH_GSUB 4     /* the march stops at the eliminated values g; the
                                divergence and projection kernels substitute u* */
CH3D_API int ch3d_path_flags(ch3d_ctx* ctx, int* flags);

#ifdef __cplusplus
}
#endif
#endif /* CH3D_H_ */
