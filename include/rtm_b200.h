/*
 * rtm_b200.h - C ABI of the B200 reverse-time-migration propagation engine.
 *
 * This is the drop-in boundary for bgprtm's propagation path.  Every entry
 * point takes plain pointers and sizes, returns an int status (0 = ok,
 * negative = rtm_status), never aborts and never throws.  Host arrays are
 * copied; device state is owned by the handle.  A handle is bound to the
 * CUDA device that was current at rtm_create and to one internal stream; it
 * is not thread-safe, but several handles (shots) may live side by side.
 *
 * Volume layout everywhere is the reference's: z fastest, then x, then y,
 * element (ix, iy, iz) at ((iy * nx + ix) * nz + iz)
 * (bgprtm/FdEngine.h:41-43, bgprtm/Propagator.cpp:528).
 *
 * Reference seams replaced (bgprtm, C++ objects, no C ABI of their own):
 *   KernelCPU::KernelCPU/setModel/setBoundary   -> rtm_create, rtm_set_model
 *       (bgprtm/KernelCPU.h:19-27)
 *   KernelCPU::ISO / VTI / TTI                  -> rtm_kernel
 *       (bgprtm/KernelCPU.h:29-33, bgprtm/KernelCPU.cpp:93-174)
 *   KernelCPU::cleanPMLMemory, Wavefield::cleanMemory -> rtm_reset
 *       (bgprtm/KernelCPU.h:35, bgprtm/Wavefield.cpp:144-170)
 *   Propagator::update2nd (+ Q branch)          -> rtm_update2nd
 *       (bgprtm/Propagator.cpp:1764-1818)
 *   Propagator::Vel2                            -> inside rtm_set_model
 *       (bgprtm/Propagator.cpp:711-742)
 *   Q::updateCq                                 -> rtm_set_q_coeffs
 *       (bgprtm/Q.cpp:310-318)
 *   Receiver::apply / apply_src                 -> rtm_inject
 *       (bgprtm/Receiver.cpp:1204-1279, 477-507)
 *   ExtractReceiverData::extract / extract_value -> rtm_extract
 *       (bgprtm/ExtractReceiverData.cpp:199-262, bgprtm/Receiver.cpp:394-426)
 *   Util::CompactOrmsbySpreadCoeff              -> rtm_spread_coeffs
 *       (bgprtm/Util.cpp:317-397, bgprtm/Receiver.cpp:291-363)
 *   Wavefield::swapPointers                     -> rtm_swap
 *       (bgprtm/Wavefield.cpp:175-178)
 *   WaveFieldCompress::compress / uncompress    -> rtm_c16_compress / rtm_c16_uncompress
 *       and snapshot store                     -> rtm_snapshot_store
 *       (bgprtm/WaveFieldCompress.cpp:107-236)
 *   ImagingCorrelator::crossone + ImagingCondition::applyTape -> rtm_image_accumulate
 *       (bgprtm/ImagingCorrelator.cpp:180-194, bgprtm/ImagingCondition.cpp:180-226)
 *   Propagator::modelling / migration time loops -> rtm_modelling / rtm_migration
 *       (bgprtm/Propagator.cpp:1054-1155, 1157-1260)
 *   PhaseCorrection::applyForward / applyBackward -> rtm_phase_correct
 *       (bgprtm/PhaseCorrection.cpp:117-235)
 */
#ifndef RTM_B200_H
#define RTM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rtm_status {
  RTM_OK = 0,
  RTM_ERR_ARG = -1,         /* bad argument (null pointer, size out of range) */
  RTM_ERR_STATE = -2,       /* call out of order (e.g. no model set) */
  RTM_ERR_CUDA = -3,        /* CUDA runtime error (message via rtm_last_error) */
  RTM_ERR_NOMEM = -4,       /* device allocation failed */
  RTM_ERR_UNSUPPORTED = -5, /* configuration not built */
  RTM_ERR_NONFINITE = -6,   /* NaN/Inf detected in an input or the state */
  RTM_ERR_TIMEOUT = -7      /* a bounded device wait gave up */
} rtm_status;

/* FD::FD, FD::CFD, FD::FFTWR2C and FD::FFTWR2R (pseudo-spectral: FFT or
 * cosine / sine transform derivative along each axis, PML along the
 * derivative's own axis only, so pml3d is ignored; bgprtm/FdEngine_r2c.cpp,
 * bgprtm/FdEngine_r2r.cpp), FD::CFD_BATCH (the Derivative path of
 * Propagator::kernel, bgprtm/Propagator.cpp:901-943: compact FD through
 * Derivative_cfd, Boundary's per-axis PML so pml3d is ignored, the
 * divergence-pass plan of iswitch), FD::FFTV and FD::SINCOS (the same
 * Derivative path with Derivative_fftv's spectral first derivative and
 * Derivative_sincos's cosine / sine transform pair, bgprtm/Derivative_fftv.cpp,
 * bgprtm/Derivative_sincos.cpp; libfftv, which implements both, is not in the
 * reference tree: here the plain spectral derivative (every bin below Nyquist
 * times i k, an even line's Nyquist bin zeroed) and the FFTWR2R line
 * operators) */
enum {
  RTM_ENGINE_FD8 = 0,
  RTM_ENGINE_CFD = 1,
  RTM_ENGINE_R2C = 2,
  RTM_ENGINE_R2R = 3,
  RTM_ENGINE_CFDB = 4,
  RTM_ENGINE_FFTV = 5,
  RTM_ENGINE_SINCOS = 6
};
enum { RTM_ISO = 1, RTM_VTI = 2, RTM_TTI = 3 };       /* ModelType (bgprtm/Model.h:13) */
enum { RTM_FORWARD = 0, RTM_BACKWARD = 1 };           /* PROP::Direction */
enum { RTM_SNAP_FP32 = 0, RTM_SNAP_C16 = 1, RTM_SNAP_FP16S = 2, RTM_SNAP_AE = 3 };
enum { RTM_IC_IMAGE1 = 0, RTM_IC_INVERSION = 1 }; /* ImagingCorrelator options IMAGE1, INVERSION */
enum {
  RTM_FIELD_W0 = 0,  /* current/next wavefield (written by the step) */
  RTM_FIELD_W1 = 1,  /* previous wavefield (read by the stencil) */
  RTM_FIELD_VEL = 2, /* (v*dt)^2 after Vel2 */
  RTM_FIELD_IMAGE = 3,
  RTM_FIELD_INVQ = 4, /* invQ after the Vel2 correction */
  RTM_FIELD_ILLUM = 5 /* source illumination, or its damping factor after rtm_illum_compensate */
};

typedef struct rtm_dims {
  int nx, ny, nz;   /* grid incl. PML; nx, nz >= 9, 1 <= ny <= 65535 */
  float dx, dy, dz; /* spacing (m) */
  float dt;         /* time step (s) */
} rtm_dims;

typedef struct rtm_config {
  int engine;         /* RTM_ENGINE_FD8 / _CFD / _R2C / _R2R / _CFDB / _FFTV / _SINCOS */
  int model_type;     /* RTM_ISO, RTM_VTI, RTM_TTI */
  int use_q;          /* visco-acoustic memory variables (Q::order terms) */
  int q_order;        /* number of memory variables, default 4 */
  int nbnd[6];        /* PML widths: x1, x2, y1, y2, z1, z2 (0 = none) */
  float vmax;         /* PML profile velocity (m/s) */
  float pml_eps;      /* PML reflection target, default 1e-3 */
  int pml3d;          /* default 1: PML on the summed operator / cross terms */
  float pml3d_scaler; /* cross-term damping scale, default 0.3 */
  int top_pml;        /* default 1; 0 = free surface top (no z1 PML) */
  int state_fp16;     /* 0: FP32 wavefield state (default); 1: FP16 w0 / w1 with a per-y-slab scale
                         (stencils, PML, Q memory and image in FP32), FD8 VTI / TTI (+Q) only, loop
                         drivers only (the stepwise seam calls return RTM_ERR_UNSUPPORTED) */
  int kernel_variant; /* 0: auto (FD8: 4 z cells per thread with TMA rings when nz % 4 == 0 and,
                         for VTI / TTI, the state is FP32; the autotuner picks among all FD8
                         kernels; compact FD: line solves and pointwise epilogues with TMA x / y
                         tiles when nz % 4 == 0, else register-streamed x / y lines; the
                         autotuner may pick any compact-FD form; FFTWR2R / SINCOS / FFTWR2C /
                         FFTV: line operators on the tensor cores, split TF32, where nz % 4 == 0
                         and lines have at most 512 points), 1: one cell per thread / plain
                         staged tiles (FFTWR2R / SINCOS: FP32 cuBLAS line products; FFTWR2C /
                         FFTV: cuFFT transforms),
                         2: compact-FD x / y TMA tiles, ISO FD8 one-cell TMA plane pipeline,
                         3: FD8 4 z cells per thread with TMA rings, 4: ISO FD8 4 z cells per
                         thread with register prefetch, 5: compact FD with
                         register-streamed x / y lines, 6: compact FD segment-parallel (line
                         solves with the PML, scaling and update fused into them) with plain tile
                         loads, 7: as 3 with the visco-acoustic update loading its Q memory
                         itself instead of from the divergence pass's TMA ring, 8: compact FD
                         segment-parallel with TMA tile loads where the tensor maps can be made,
                         9: as 0 with each compact-FD z line solve carrying the interior cells of
                         the pointwise epilogue that follows it (the PML cells stay separate
                         launches), 10: as 0 with the compact-FD x / y line solves by the
                         pipelined persistent TMA kernel (the 4-cell and segment-parallel
                         variants fall back when they do not apply) */
  int use_rho;        /* density model (KernelCPU::setModel's rho, bgprtm/KernelCPU.cpp:76-78):
                         the gradient is divided by rho (KernelCPU::divideRho) and the divergence
                         accumulates vel * rho (bgprtm/FdEngine_fd.cpp:411, 437, 463); ISO then takes
                         the first-derivative passes (bgprtm/KernelCPU.cpp:128).  FD8 density runs
                         use the one-cell passes; not with state_fp16 */
  int q_bf16;         /* use_q: the memory variables wq[2][L][N] stored as bfloat16 (read and
                         rounded back each step; the update arithmetic stays FP32): half their
                         HBM traffic, the largest share of a TTI + Q step */
} rtm_config;

typedef struct rtm_handle rtm_handle;

/* Fills the reference's defaults (pml_eps 1e-3, pml3d 1, scaler 0.3, q_order 4). */
void rtm_config_default(rtm_config *cfg);

/* Reference seam: KernelCPU(nx,ny,nz,dx,dy,dz,engine,nThreads) + setBoundary(...)
 * (bgprtm/KernelCPU.h:19,27; bgprtm/FdEngine.cpp:108-182).  Allocates all device
 * state (wavefields, PML memory, Q memory) and builds the FD / CFD tables and
 * the PML profile in FP64. */
int rtm_create(const rtm_dims *dims, const rtm_config *cfg, rtm_handle **out);
int rtm_destroy(rtm_handle *h);

/* Text of the last error on this handle (or of the last failed create when h is NULL). */
const char *rtm_last_error(const rtm_handle *h);

/* Q::updateCq (bgprtm/Q.cpp:310-318): cq0, cq[q_order], wq[q_order].  Must
 * precede rtm_set_model when use_q. */
int rtm_set_q_coeffs(rtm_handle *h, float cq0, const float *cq, const float *wq);

/* KernelCPU::setModel(vel, rho, del, eps, pjx, pjy) + Propagator::Vel2
 * (bgprtm/KernelCPU.cpp:76-83, bgprtm/Propagator.cpp:711-742).  vel is
 * velocity in m/s; it is converted to (v*dt)^2 on the device (Q-corrected when
 * use_q).  rho (density, > 0) is required when the configuration sets use_rho
 * and must be NULL otherwise; eps/del are needed for VTI/TTI, pjx/pjy for TTI,
 * invq (1/Q) for use_q; others may be NULL. */
int rtm_set_model(rtm_handle *h, const float *vel, const float *rho, const float *eps, const float *del,
                  const float *pjx, const float *pjy, const float *invq);

/* Zero wavefields, PML memory, Q memory and the extracted traces
 * (Wavefield::cleanMemory + KernelCPU::cleanPMLMemory). */
int rtm_reset(rtm_handle *h);

/* One application of the spatial operator: w0 -= (v dt)^2 * L[w1]
 * (KernelCPU::ISO/VTI/TTI with PML, bgprtm/KernelCPU.cpp:93-174). */
int rtm_kernel(rtm_handle *h);

/* Leapfrog w0 = 2 w1 - w0, or the Q form (bgprtm/Propagator.cpp:1767-1818). */
int rtm_update2nd(rtm_handle *h);

/* Swap w0/w1 and the Q memory halves (Wavefield::swapPointers). */
int rtm_swap(rtm_handle *h);

/* Separable spread kernel of one trace along one axis
 * (Util::CompactOrmsbySpreadCoeff with nlimit, bgprtm/Util.cpp:317-397, then
 * the edge taper of Receiver::spreadCoeffs, bgprtm/Receiver.cpp:291-303).
 * n: grid size on the axis; x: fractional grid index; k1, k2: pass/cut
 * wavenumbers (fraction of Nyquist*0.5, 0 < k1 <= k2 <= 0.5); *nlimit: in =
 * kernel capacity (2*spread), out = used length; coeff[nlimit]; ntaper: edge
 * taper length (0 = none).  Returns the first grid index in *off. */
int rtm_spread_coeffs(int n, float x, float k1, float k2, int *nlimit, int dipole, int ntaper,
                      float *coeff, int *off);

/* Receiver FK true-amplitude / deghost spreading, space domain
 * (Receiver::spread_sdomain, bgprtm/Receiver.cpp:851-1010, the default of
 * Receiver::spread): the traces are spread onto the (ny, nx) receiver grid with
 * their separable kernels, transformed over (y, x, t), filtered per bin
 * (obliquity sqrt(1 - kh^2 / k^2) when trueamp; with deghost 1 / (2 sin(kz z))
 * capped at 1 / ghost_threshold, the low-cut ramp, a quarter-period phase
 * turn signed by side) and transformed back.  The result, one trace per grid
 * column, is what the injection then spreads in z (a trace set with x / y
 * kernels of length one).  Host in, host out, on the current device. */
typedef struct rtm_fk_args {
  int nx, ny, nt, ntfft; /* receiver grid (x, y), samples per trace, time FFT length (>= nt;
                            libfftv::padfftv is not in the reference tree) */
  float dt, dx, dy;      /* sample interval (s), grid spacing (m) */
  float vsurf, z;        /* surface velocity (m/s), mean receiver depth below the surface (m) */
  int trueamp, deghost;  /* obliquity factor; ghost removal */
  int side;              /* -1 receivers (backward propagation), +1 sources */
  float flcut, flpass;   /* souLowCut / souLowPass (Hz): low-cut ramp, with deghost */
  float ghost_threshold; /* ghost_zerofreq_threshold (reference default 0.1) */
  float khpass, khcut;   /* spread kernel band, as rtm_spread_coeffs */
  int nlimit;            /* spread kernel length cap (2 x spread size) */
  int domain;            /* 0: space domain (fk_domain SDOMAIN, the reference default);
                            1: wavenumber domain (KDOMAIN, Receiver::spread_kdomain,
                            bgprtm/Receiver.cpp:641-849; nx > 1, khpass < khcut) */
  float fmax;            /* KDOMAIN: highest data frequency (Hz), scales the ghost threshold */
} rtm_fk_args;
/* xy [nr][2]: fractional grid indices (x, y); traces [nr][nt]; out [ny][nx][nt] */
int rtm_fk_spread(const rtm_fk_args *a, int nr, const float *xy, const float *traces, float *out);

/* Time-dispersion / phase correction of traces (PhaseCorrection,
 * bgprtm/PhaseCorrection.h:11-25, bgprtm/PhaseCorrection.cpp:14-235): the
 * constructor's arguments and the global parameters it reads, then
 * applyForward (apply 1) or applyBackward (apply 2) on ntr traces of nt
 * samples.  The correction table exp(i phs(iw, it)) * factor(iw) of init()
 * (:62-115) is built on the host in the reference's float order; the table
 * transforms (fft_dft's time sum, dft_fft's frequency sum) run as one tiled
 * FP32 product kernel, the plain transforms on cuFFT.  libfftv (fft_r2c_fd,
 * fft_c2r_bd, padfftv) is absent from the reference tree; its conventions
 * are inferred from these call sites: forward unnormalised with exp(+i w t),
 * the Nyquist bin packed into bin 0's imaginary part (cleared by the
 * reference), backward the unnormalised Hermitian sum with exp(-i w t);
 * ntfft is the caller's (even, >= nt).
 * Output: apply 1 writes [ntr][nt]; apply 2 writes [ntr][nt_dft] (nt_dft =
 * nt_out when resampling, else nt).  scaler (apply 2) multiplies the first
 * nt_out samples of each output trace when nt_out > 0 (:138-139; every
 * reference call passes one trace).  Refused (RTM_ERR_ARG): apply 1 on a
 * direction other than FWD (:117), resampling with apply 1 or on a dft_fft
 * path (:182), the no-op (no tdsp, w_pow 0, phase 0) with resampling (:130),
 * fft_dft without the table when ntfft < nt_out (the reference leaves the
 * output's tail unwritten, :185-186).  Host in, host out, on the current
 * device. */
typedef struct rtm_phase_args {
  int nt;                   /* samples per input trace */
  float dt, Dt, t0, fmax;   /* sample interval, propagation dt (0: no dispersion term), start time, max frequency */
  int direction;            /* PhaseCorrection::DIRECTION: 0 NONE, 1 FWD, 2 BWD */
  float w_pow, phase_deg;   /* (i w)^w_pow magnitude factor, constant phase rotation (degrees) */
  int do_tdsp;              /* 0: no table (tdsp_correction forced to 0) */
  int nt_out;               /* resampling: output samples (> 0 with dt_out > 0), else -1 */
  float dt_out, t0_out;     /* resampling: output interval and start time */
  int ntfft;                /* time FFT length (libfftv::padfftv stand-in), even, >= nt */
  int tdsp_correction;      /* global tdsp_correction (reference default 2) */
  int skip_tdsp_correction; /* global skip_tdsp_correction bits (1 FWD, 2 BWD) */
  float tdsp_acos_ratio;    /* global tdsp_acos_ratio (0: sin form, 1: acos form) */
  int skip_jacobian;        /* global tdsp_skip_jacobian */
  int transform;            /* 0: by direction; 1: tdsp_force_fftdft; 2: tdsp_force_dftfft */
} rtm_phase_args;
int rtm_phase_correct(const rtm_phase_args *a, int apply, int ntr, const float *in, float *out, float scaler);

/* The FFTWR2R first derivative along one axis of n points with spacing d as
 * the row-major n x n matrix D the engine applies to every line (out_t =
 * sum_u D[t][u] x_u): FdEngine_r2r::fftderiv1_r2r, bgprtm/FdEngine_r2r.cpp:73-102;
 * isign +1 (gradient pass) or -1 (divergence pass).  Host only. */
int rtm_r2r_line_matrix(int n, float d, int isign, float *D);

/* Traces injected into w0 each step (Receiver::apply, no FK/true-amp path):
 * w0[c] += traces[r][it] * scaler * kx[r][ix] * ky[r][iy] * kz[r][iz] * (v dt)^2[c]
 * Kernels are packed with fixed strides lx, ly, lz per trace; off3/len3 are
 * [ntr][3] (x, y, z) first index and used length.  scaler is the reference's
 * dt_dxyz = 1/(dx*dy*dz) times Receiver::apply's scaler0.  Copies everything. */
int rtm_set_injection(rtm_handle *h, int ntr, int lx, int ly, int lz, const int *off3,
                      const int *len3, const float *kx, const float *ky, const float *kz,
                      const float *traces, int nt, float scaler);

/* Receivers read from w0 (ExtractReceiverData::extract with template receivers):
 * out[r][jt] = sum kx*ky*kz*w0 over the trace's kernel box. */
int rtm_set_extraction(rtm_handle *h, int ntr, int lx, int ly, int lz, const int *off3,
                       const int *len3, const float *kx, const float *ky, const float *kz,
                       int nt_out);

/* Apply injection sample it (no-op outside [0, nt)). */
int rtm_inject(rtm_handle *h, int it);
/* Extract receivers into sample jt (no-op outside [0, nt_out)). */
int rtm_extract(rtm_handle *h, int jt);
/* Copy extracted traces [ntr][nt_out] to host. */
int rtm_get_traces(rtm_handle *h, float *dst);

/* Snapshot store for the source wavefield: nslots slots of format fmt
 * (RTM_SNAP_FP32 uncompressed, RTM_SNAP_C16 = the reference's COMPRESS_16
 * codec, bit-exact, RTM_SNAP_FP16S = FP16 with a per-y-slab scale,
 * RTM_SNAP_AE = the learned compressor attached by rtm_set_compressor:
 * 64 BF16 latent values + 1 scale per 8^3 block, 15.5:1). */
int rtm_snapshot_setup(rtm_handle *h, int fmt, int nslots);
/* Store w0 into slot (WaveFieldCompress::compress + CacheFile write). */
int rtm_snapshot_store(rtm_handle *h, int slot);
/* Decode slot into dst (host, N floats) with the reference's decode tapers. */
int rtm_snapshot_load(rtm_handle *h, int slot, float *dst);
/* Snapshot offload (CacheFile / AsyncIO / WaveFieldHolder spill,
 * bgprtm/CacheFile.cpp:32-109, bgprtm/WaveFieldHolder.cpp:50-77): after
 * rtm_snapshot_setup, moves the slots to pinned host memory and keeps nstage
 * (2..8) device slots that stage them; the forward loop copies each stored
 * snapshot to the host while the next steps run, the backward loop fetches
 * slots ahead of the imaging condition.  Clears the slots; nstage = 0 returns
 * to device slots.  FP32, COMPRESS_16 and FP16 formats. */
int rtm_snapshot_offload(rtm_handle *h, int nstage);
/* Bytes of one snapshot slot of format fmt on this handle (the learned
 * format with the current FP16 fallback setting); allocates nothing. */
int rtm_snapshot_slot_bytes(rtm_handle *h, int fmt, size_t *bytes);
/* Snapshot slot window: the loops put the snapshot of step it in slot
 * it / interval - first and skip steps whose slot falls outside
 * [0, nslots); clears the stored flags; the imaging condition's time taper
 * still follows the snapshot's number in the shot (slot + first).
 * rtm_snapshot_setup sets it to 0.  With checkpoints
 * (below) a backward pass over a long shot images one segment at a time
 * from slots that hold only that segment's snapshots. */
int rtm_snapshot_window(rtm_handle *h, int first);
/* Checkpoints of the propagation state, the store / recompute alternative to
 * spilling snapshots (the reference spills them to a cache file,
 * bgprtm/CacheFile.cpp:32-109; it has no checkpoints): nckpt device slots
 * that each hold the wavefields w0 / w1 (FP16 state: codes, slab scales and
 * maxima), the Q memory of both time levels and every PML memory array;
 * *bytes_each (optional) receives the bytes per slot.  Save / load copy on
 * the engine's stream: loading slot k and running the loop from step it
 * reproduces, bit for bit, what the loop computed from the step at which
 * slot k was saved.  The source / receiver traces and the image are not part
 * of the state. */
int rtm_checkpoint_setup(rtm_handle *h, int nckpt, size_t *bytes_each);
int rtm_checkpoint_save(rtm_handle *h, int k);
int rtm_checkpoint_load(rtm_handle *h, int k);

/* Imaging condition set-up: ntaper_t source time-taper snapshots, ntaper_z
 * depth-taper cells (ImagingCondition::calTapes), edge_taper=1 applies the
 * snapshot decode tapers (20 cells x/y, 10 z) to both fields
 * (WaveFieldCompress::uncompress16).  Clears the image. */
int rtm_image_setup(rtm_handle *h, int ntaper_t, int ntaper_z, int edge_taper);
/* image += T(src[slot]) * T(w0), zero lag, Kahan-compensated FP32. */
int rtm_image_accumulate(rtm_handle *h, int slot);
/* Imaging condition of the backward loop and of rtm_image_accumulate
 * (ImagingCondition::getImagingOption, bgprtm/ImagingCondition.cpp:151-160):
 * RTM_IC_IMAGE1 (default) the zero-lag correlation s r fused into the next step;
 * RTM_IC_INVERSION (the reference's default LowcutFilter) s r - grad^ s . grad^ r with
 * the normalised k-domain derivatives of both tapered fields
 * (ImagingCorrelator::inversion1, bgprtm/ImagingCorrelator.cpp:374-424), computed with
 * cuFFT at each imaging step.  The first INVERSION call creates the FFT plans and 4
 * volumes + 3 spectra of scratch (call it before any stream capture). */
int rtm_image_condition(rtm_handle *h, int option);
/* Double-grid IMAGE1 (ImagingCondition with ic_double_z / _x / _y = 2; stackImageInterp,
 * applyFFTV and interp, bgprtm/ImagingCondition.cpp:104-141, 169-178, 1084-1111;
 * ImagingCorrelator::imaging1 and interleave2d / interleave3d,
 * bgprtm/ImagingCorrelator.cpp:363-372, 440-507): at every imaging step both tapered
 * fields are high-cut along each doubled axis (above high_z / high_xy of the Nyquist
 * wavenumber, cosine roll-off; the reference's defaults are 0.9 and 0.7), half-shifted
 * into the 2, 4 or 8 copies that sit on the doubled grid's sub-lattices (line FFTs:
 * value at x + d/2), and copy i of the source is correlated with copy i of the receiver
 * into image cube i.  The filters restate libfftv's HIGHTAPE / SHIFTHALF from their use
 * (libfftv is not in the reference tree).  Factors (z, x, y): (2, 1, 1) or (2, 2, 1) on
 * 2-D grids, (2, 2, 2) on 3-D grids; (1, 1, 1) turns it off.  IMAGE1 only (not with
 * RTM_IC_INVERSION).  Replaces the fused image term of the backward loop and of
 * rtm_image_accumulate while on; rtm_image_setup clears its cubes.  Allocates the
 * line-FFT plans and 2 * nloop + 2 * nloop volumes (call it before any stream capture). */
int rtm_image_double(rtm_handle *h, int ndbl_z, int ndbl_x, int ndbl_y, float high_z, float high_xy);
/* The double-grid image on the doubled grid [ny * ndbl_y][nx * ndbl_x][nz * ndbl_z]
 * (ImagingCorrelator::interleave); dst holds nloop * nx * ny * nz floats. */
int rtm_get_image_double(rtm_handle *h, float *dst);
/* The source illumination interpolated onto the doubled grid
 * (ImagingCondition::interpIllum, bgprtm/ImagingCondition.cpp:759-808, its arithmetic
 * and write order); needs rtm_illum_setup. */
int rtm_get_illum_double(rtm_handle *h, float *dst);
/* Source illumination (ImagingCondition::calIllum, bgprtm/ImagingCondition.cpp:143-149):
 * on = 1 allocates and zeroes a volume that every later imaging-condition term adds the
 * squared source value to (after the time / depth and edge tapers); on = 0 stops. */
int rtm_illum_setup(rtm_handle *h, int on);
/* Shot illumination compensation (ShotIllumComp, ImagingCondition::computeDamping +
 * applyDamping, bgprtm/ImagingCondition.cpp:600-689): box-smooths the illumination
 * (half widths smooth_xy, smooth_z; avgVolume3D, both 0 = no smoothing), turns it into the
 * damping factor 1 / (avg (a + damp_weight e^-a)), a = illum / avg, avg = mean^amp_damping,
 * with 10-cell x / y edge tapers, and multiplies the image by it.  Reference defaults:
 * 10, 10, 1.0, 0.07. */
int rtm_illum_compensate(rtm_handle *h, int smooth_xy, int smooth_z, float amp_damping, float damp_weight);

/* Propagator::modelling loop (bgprtm/Propagator.cpp:1099-1153): for it in
 * [0, nts): kernel, update2nd, inject(it + it_shift), extract(it / ntratio)
 * when it % ntratio == 0, swap.  Fused kernels; time loop in a CUDA graph. */
int rtm_modelling(rtm_handle *h, int nts, int it_shift, int ntratio);

/* Propagator::migration loop (bgprtm/Propagator.cpp:1210-1255).
 * dir = RTM_FORWARD: it = 0 .. it_end-1, inject(it + it_shift), store slot
 *   it/interval when it % interval == 0 and the slot exists.
 * dir = RTM_BACKWARD: it = it_begin down to it_end+1, inject(it - it_shift),
 *   image += src[it/interval] * w0 when it % interval == 0 and that slot was
 *   stored (the zero-lag correlation fused into the backward step). */
int rtm_migration(rtm_handle *h, int dir, int it_begin, int it_end, int it_shift, int interval);

/* Copy a field (RTM_FIELD_*) of N floats to / from host memory. */
int rtm_get(rtm_handle *h, int field, float *dst);
int rtm_put(rtm_handle *h, int field, const float *src);

/* The reference's COMPRESS_16 codec on host buffers, run on the device
 * (bit-exact with WaveFieldCompress::compress16/uncompress16).  out holds
 * (nx*nz + 2) * ny uint16 values, ny <= 65535.  uncompress applies the decode
 * tapers. */
int rtm_c16_compress(const float *in, unsigned short *out, int nx, int ny, int nz);
int rtm_c16_uncompress(const unsigned short *in, float *out, int nx, int ny, int nz);

/* No counterpart in the reference.  COMPRESS_16 encoding of a wavefield that is
 * already on the device, for callers that cannot allocate GPU memory (a host
 * program that carves all of HBM up front with its own pool allocator, or a
 * thread that must not wait on the allocator).  d_in: nx*ny*nz floats,
 * d_out: (nx*nz + 2)*ny uint16, both device memory of the current device, same
 * layout and bit-exact codes as rtm_c16_compress.  Allocates nothing: its
 * scratch (one float per y slab) is a fixed array of RTM_NOALLOC_MAX_SLABS
 * floats that every GPU loading the library holds until exit; ny above that
 * limit returns RTM_ERR_ARG.  The first call in a CUDA context (the runtime's
 * primary context of a device, or a context the caller made current) looks
 * the array's device address up (cudaGetSymbolAddress), so make that first
 * call before any stream capture.  Runs asynchronously on `stream` (a
 * cudaStream_t, NULL = default stream).  All calls on a device share the
 * scratch, which keeps the last call's contents: calls that can overlap on the
 * GPU (different streams without ordering) race, so order or serialise them. */
#define RTM_NOALLOC_MAX_SLABS 65535
int rtm_c16_compress_noalloc(const float *d_in, unsigned short *d_out, int nx, int ny, int nz, void *stream);

/* Device time of the last rtm_modelling / rtm_migration call (ms, CUDA events). */
int rtm_last_loop_ms(rtm_handle *h, float *ms);
/* ---- Learned snapshot compressor ------------------------------------------
 * A 3-D convolutional autoencoder on 8^3-cell blocks (4 encoder + 4 decoder
 * layers, 16 channels, 512 cells -> 64 BF16 latent values + the block's max |w|),
 * trained and run on the GPU with BF16 tensor-core GEMMs and FP32
 * accumulation.  Replaces WaveFieldCompress (bgprtm/WaveFieldCompress.cpp
 * compress/uncompress) for the forward-wavefield snapshots when attached to a
 * handle; the FP32 / COMPRESS_16 stores stay available as the fallback.
 * Blocks on the host are [n][512] floats, each scale-normalised (max |v| = 1)
 * and in Morton order within the block (bit triples z y x from the least
 * significant bit).  Parameters: rtm_ae_nparams() floats, layer by layer
 * W [K][N] then bias [N]. */
typedef struct rtm_ae rtm_ae;
int rtm_ae_nparams(void);
int rtm_ae_create(rtm_ae **out);
int rtm_ae_destroy(rtm_ae *a);
int rtm_ae_set_params(rtm_ae *a, const float *params);
int rtm_ae_get_params(rtm_ae *a, float *params);
/* MSE loss of the reconstruction of n host blocks and its gradient
 * (grads may be NULL); no update. */
int rtm_ae_loss_grad(rtm_ae *a, const float *blocks, int n, float *loss, float *grads);
/* One Adam step (learning rate lr) on a batch of n host blocks; returns the
 * batch loss before the step. */
int rtm_ae_train_step(rtm_ae *a, const float *blocks, int n, float lr, float *loss);
/* Reconstruction [n][512] (and the FP32 latents [n][64] when latent != NULL). */
int rtm_ae_reconstruct(rtm_ae *a, const float *blocks, int n, float *out, float *latent);
/* Device volume (z fastest) <-> latents [nb][64] as bfloat16 (128 bytes per
 * block) + scales [nb] (float), nb = the 8^3 blocks covering the volume
 * (zero-padded); on `stream` (NULL = default). */
int rtm_ae_compress_volume(rtm_ae *a, const float *d_vol, int nx, int ny, int nz, void *d_latent, float *d_scales,
                           void *stream);
int rtm_ae_decompress_volume(rtm_ae *a, const void *d_latent, const float *d_scales, int nx, int ny, int nz,
                             float *d_vol, void *stream);
/* Attach a compressor to a handle (same device) for RTM_SNAP_AE snapshots. */
int rtm_set_compressor(rtm_handle *h, rtm_ae *a);
/* Fallback of learned snapshots to a plain store for the blocks the code
 * represents worst, the high-energy ones: each RTM_SNAP_AE slot also keeps, as
 * FP16 values of v / block scale, the 8^3 blocks whose scale exceeds tau x the
 * slot's largest, largest first, at most ceil(max_fraction x blocks) of them;
 * decoding overwrites those blocks.  max_fraction = 0 turns it off (default).
 * Clears existing RTM_SNAP_AE slots (their size changes) and their host
 * offload (call rtm_snapshot_offload again).  No counterpart in the
 * reference (its WaveFieldCompress has no learned code). */
int rtm_set_compressor_fallback(rtm_handle *h, float tau, float max_fraction);

/* ---- Batched small shots (many shots, one persistent launch per step) ----
 * A batch steps several FD8 handles (no Q) of different grids and step counts
 * together: all ISO (each time step one persistent kernel over the column
 * tiles of every active shot) or all VTI, or all TTI (each step two persistent
 * kernels, the gradient and the divergence pass of the one-cell kernels; no
 * density, FP32 state), then one batched injection and one batched extraction
 * launch; the time loop runs as CUDA graphs.  Each handle must have its model,
 * injection (and, optionally, extraction) set and be reset.
 * No reference counterpart: bgprtm runs one shot per process
 * (bgprtm/Propagator.cpp:1054-1260 per shot). */
typedef struct rtm_batch rtm_batch;
int rtm_batch_create(rtm_handle *const *shots, int nshots, rtm_batch **out);
int rtm_batch_destroy(rtm_batch *b);
/* rtm_modelling(shots[s], nts[s], it_shift, ntratio) for every shot at once:
 * same wavefields and traces (receiver sums may differ in the last bit from a
 * handle's grouped extraction). */
int rtm_batch_modelling(rtm_batch *b, const int *nts, int it_shift, int ntratio);
/* Device time of the last rtm_batch_modelling (ms). */
int rtm_batch_last_ms(rtm_batch *b, float *ms);
/* Times `steps` batched steps for each tile width / y-segment length the
 * batched kernel offers, keeps the fastest and returns its index; zeroes the
 * shots' wavefields, PML memory and traces (as rtm_reset). */
int rtm_batch_autotune(rtm_batch *b, int steps, int *choice);

/* Failure detection.  rtm_check_finite scans field RTM_FIELD_W0 / W1 / IMAGE on
 * the device and sets *nonfinite to 1 when it holds a NaN or an infinity (an
 * unstable model or dt), else 0.  RTM_ERR_ARG for a field the handle does not
 * hold (the image before rtm_image_setup).  No reference counterpart: bgprtm
 * never checks its wavefields. */
int rtm_check_finite(rtm_handle *h, int field, int *nonfinite);
/* Self-test of the engine's bounded device waits: launches one kernel whose
 * mbarrier wait can never complete; the wait gives up after its poll limit,
 * raises the device flag, and the call returns RTM_ERR_TIMEOUT with the
 * context still usable.  Any other return value is a failure.  No reference
 * counterpart. */
int rtm_selftest_bounded_wait(rtm_handle *h);
/* Autotuner: times `steps` fused steps of every launch shape this handle's
 * kernels offer (ISO FD8: 4-z-cell kernels with TMA rings or register
 * prefetch at several tile widths, prefetch depths and y segments, and the
 * one-cell TMA plane pipeline; tile width of the FD8 gradient / divergence
 * passes; register-streamed or TMA-tiled x / y line solves for compact FD),
 * keeps the fastest, returns its index in *choice, then zeroes the wavefields
 * and PML memory (as rtm_reset). */
int rtm_autotune(rtm_handle *h, int steps, int *choice);
/* Candidate `idx` of the last rtm_autotune: desc[0] kernel family (0 one cell
 * per thread / FD8 two-pass / compact FD, 1 ISO 4 z cells with register
 * prefetch, 2 ISO 4 z cells with TMA rings, 3 ISO one-cell TMA pipeline,
 * 4 FD8 VTI / TTI 4 z cells with TMA rings),
 * desc[1] its tile width or shape index, desc[2] its y segment (0: default),
 * desc[3] the compact-FD form (0 streamed, 1 TMA or 2 plain x / y tiles of the
 * split pipeline, 3 / 4 segment-parallel with TMA / plain tile loads); *ms the
 * time of its `steps` steps.
 * RTM_ERR_ARG when idx is out of range. */
int rtm_autotune_result(rtm_handle *h, int idx, int desc[4], float *ms);

/* Kernels launched by the last rtm_modelling / rtm_migration call. */
int rtm_last_loop_launches(rtm_handle *h, long long *n);

/* Kernel kinds of the per-kernel profile. */
enum {
  RTM_K_ISO = 0,       /* ISO FD8 fused step */
  RTM_K_GRAD = 1,      /* FD8 gradient pass (VTI/TTI) */
  RTM_K_DIV = 2,       /* FD8 divergence pass */
  RTM_K_CFD_Z = 3,     /* compact-FD z-line solves */
  RTM_K_CFD_X = 4,     /* compact-FD x-line solves */
  RTM_K_CFD_Y = 5,     /* compact-FD y-line solves */
  RTM_K_CFD_GEPI = 6,  /* compact-FD gradient epilogue (PML, scaling) */
  RTM_K_CFD_DEPI = 7,  /* compact-FD divergence epilogue (PML, update) */
  RTM_K_INJECT = 8,
  RTM_K_EXTRACT = 9,
  RTM_K_SLAB = 10,     /* per-slab max of the 16-bit snapshot formats */
  RTM_K_IO = 11,       /* standalone snapshot store / imaging condition */
  RTM_K_CFD_YF = 12,   /* compact FD, segment-parallel: fused y kernel (y gradient, scaling, y divergence part) */
  RTM_K_CFD_XF = 13,   /* compact FD, segment-parallel: fused x kernel (x divergence part, accumulation, update) */
  RTM_NKINDS = 14
};
/* on = 1: the time loops run eagerly (no CUDA graph) with CUDA events around
 * every launch, and the per-kind device time accumulates; on = 0 resets. */
int rtm_profile(rtm_handle *h, int on);
/* ms[RTM_NKINDS], count[RTM_NKINDS]: accumulated device time and launches. */
int rtm_profile_read(rtm_handle *h, double *ms, long long *count);

#ifdef __cplusplus
}
#endif
#endif /* RTM_B200_H */
