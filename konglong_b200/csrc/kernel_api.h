// kernel_api.h - argument blocks and launchers of the B200 RTM kernels.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rtm_internal.cuh"

struct rtm_ae;

namespace rtm {

// one column tile of the FD8 kernels: z tile bz (32 cells), x tile bx (tx
// cells), planes [y0, y1)
struct Tile4 {
  int bz, bx, y0, y1;  // z tile (32 cells), x tile (tx cells), planes [y0, y1)
};

struct IsoArgs {
  int nx, ny, nz, yseg;
  const float *w1;
  float *w0;
  const float *vel;
  float c2x[5], c2y[5], c2z[5];
  PmlDev pml;
  FusedIo io;
  QDev q;
};

// one shot of a batched ISO step (device array): its step arguments, its two
// wavefield buffers (w1 = wa on even steps) and its tile grid
struct IsoBatchShot {
  IsoArgs a;
  float *wa, *wb;
  int tiles_z, tiles_x, tiles_y;
  TraceDev inj, ext;  // source traces (scatter) and receivers (gathered into ext_out)
  float *ext_out;     // [ext.ntr][ext.nt]
};

// FP16 wavefield state (per-y-slab scale: value = half * scale[iy])
struct StateF16 {
  const __half *w1;     // current field, scale s1
  const float *s1;
  __half *w0;           // previous field (read, scale s0) overwritten by the new one (scale sn)
  const float *s0, *sn;
  unsigned *m0;         // per-slab max |new value| (float bits), atomically raised
};

struct GradArgs {
  int nx, ny, nz, yseg, pml3d;
  StateF16 h;           // used by the FP16-state instantiations
  const float *w1;
  float *px, *py, *pz;
  const float *eps, *del, *pjx, *pjy;
  const float *rho;  // density (null: none); one-cell passes only
  float c1x[5], c1y[5], c1z[5];
  PmlDev pml;
  FusedIo io;
};

struct DivArgs {
  int nx, ny, nz, yseg, pml3d;
  StateF16 h;
  const float *px, *py, *pz;
  const float *w1;
  float *w0;
  const float *vel;
  const float *rho;  // density (null: none); one-cell passes only
  float c1x[5], c1y[5], c1z[5];
  PmlDev pml;
  QDev q;
};

// one VTI / TTI shot of a batched two-pass step (device array): its pass
// arguments, its two wavefield buffers (w1 = wa on even steps, as in
// IsoBatchShot), its tile grid and y segment
struct AnisoBatchShot {
  GradArgs g;
  DivArgs d;
  float *wa, *wb;
  int tiles_z, tiles_x, tiles_y, yseg;
};
constexpr int kAnisoBatchTX = 8;  // tile width of the batched two-pass kernels
// one step (both passes) of every active VTI / TTI shot of a batch
void launch_aniso_fd8_batch(const AnisoBatchShot *shots, const int *start, int nactive, int total, int it, int model,
                            int ctas, cudaStream_t st);
int aniso_batch_ctas_per_sm();

// mode: 0 = operator only (w0 -= vel*L), 1 = + leapfrog update, 2 = + Q update
void launch_iso_fd8(const IsoArgs &a, int mode, int pml3d, int tx, cudaStream_t st);
// the same step with 4 z cells per thread (float4 rows; nz % 4 == 0), tile
// 32 (z) x tx (x) with tx in {8, 16, 32}
void launch_iso_fd8_v4(const IsoArgs &a, int mode, int pml3d, int tx, cudaStream_t st);
// the CTAs per SM launch_iso_fd8_v4 keeps resident (leapfrog mode)
int iso_v4_ctas_per_sm(int tx, int pml3d);
// one step of every active shot of a batch (ISO, leapfrog): shots[0..nactive)
// device array, start[] their first work items (start[nactive] = total)
void launch_iso_fd8_batch(const IsoBatchShot *shots, const int *start, int nactive, int total, int it, int pml3d,
                          int tx, int ctas, cudaStream_t st);
// the CTAs per SM the batched ISO kernel keeps resident at tile width tx
int iso_batch_ctas_per_sm(int tx, int pml3d);
// batched source injection at trace sample it_src and receiver extraction at
// sample jt, into the step-`it` output buffers of shots[0..nactive)
void launch_batch_inject(const IsoBatchShot *shots, int nactive, int max_ntr, int max_ly, int it_src, int it,
                         cudaStream_t st);
void launch_batch_extract(const IsoBatchShot *shots, int nactive, int max_ntr, int jt, int it, cudaStream_t st);
// one CTA per entry of tiles[0, ntiles) (column tiles of 32 z x tx x cells);
// non-edge tiles hold no PML cell and run without the PML code
void launch_grad_fd8(const GradArgs &a, const Tile4 *tiles, int ntiles, bool edge, int model, int tx,
                     cudaStream_t st, bool f16 = false);
void launch_div_fd8(const DivArgs &a, const Tile4 *tiles, int ntiles, bool edge, int mode, int tx, cudaStream_t st,
                    bool f16 = false);
// FP16 state: new-field scales sn[y] = max(max over |dy| <= 4 of m0 / m1, floor) * 2^-12
void launch_f16_scales(const unsigned *m0, const unsigned *m1, float *sn, int ny, float floor, cudaStream_t st);
// snapshot slab headers of the FP16 state's new field from its slab maxima
void launch_f16_slab_hdr(const unsigned *m, float *slab, uint16_t *c16, int fmt, int nx, int ny, int nz,
                         cudaStream_t st);
// FP16 state <-> FP32 volume; f32_to_f16 takes the slab max, sets the scale
// (max * 2^-12, at least floor * 2^-12) and records the max
void launch_f16_to_f32(const __half *h, const float *s, float *out, int ny, long long nxz, cudaStream_t st);
void launch_f32_to_f16(const float *in, __half *h, float *s, unsigned *m, int ny, long long nxz, float floor,
                       cudaStream_t st);
// FP16 state: scatter of every trace into h (scale s), raising the slab max m;
// gather of every receiver from h
void launch_inject_scatter_f16(const TraceDev &t, int it, __half *h, const float *s, unsigned *m, const float *vel,
                               int nx, int ny, int nz, cudaStream_t st);
void launch_extract_direct_f16(const TraceDev &t, const __half *h, const float *s, float *out, int jt, int nt_out,
                               int nx, int ny, int nz, cudaStream_t st);

// ---- TMA plane pipelines (kernels_tma.cu), nz % 4 == 0 ------------------------
bool tma_supported(int nz);
// one kernel whose bounded mbarrier wait can never complete (raises *err)
void launch_selftest_wait(int *err, cudaStream_t st);
// fp32 volume [ny][nx][nz], box (bz, bx, 1)
bool make_tmap(CUtensorMap *m, const void *base, int nx, int ny, int nz, int bz, int bx, int by = 1);
// Q memory variables [L][ny][nx][nz] (FP32 or BF16), 4-D box (bz, bx, 1, L)
bool make_tmap_q(CUtensorMap *m, const void *base, int nx, int ny, int nz, int L, bool bf16, int bz, int bx);
struct TmaShape {
  int tx, depth;  // tile width (x) and planes prefetched beyond the stencil window
};
extern const TmaShape kIsoTmaShapes[];
extern const int kIsoTmaNShapes;
bool iso_tma_init();  // shared-memory attributes (call outside any capture)
void launch_iso_fd8_tma(const IsoArgs &a, const CUtensorMap &w1, const CUtensorMap &w0, const CUtensorMap &vel,
                        int *err, int mode, int pml3d, int shape, cudaStream_t st);
// the 4-z-cells-per-thread step with TMA rings (kernels_iso4.cu): tensor maps
// with boxes (40, tx + 8) for w1 and (32, tx) for w0 / (v dt)^2.  One CTA per
// entry of a tile table (device array); `edge` tiles may hold PML cells, the
// others run a kernel compiled without the PML code.
extern const TmaShape kIso4TmaShapes[];
extern const int kIso4TmaNShapes;
bool iso_tma4_init();
int iso_tma4_ctas_per_sm(int shape, int pml3d);
void launch_iso_fd8_tma4(const IsoArgs &a, const Tile4 *tiles, int ntiles, bool edge, const CUtensorMap &w1,
                         const CUtensorMap &w0, const CUtensorMap &vel, int *err, int mode, int pml3d, int shape,
                         cudaStream_t st);

// FD8 VTI / TTI passes with 4 z cells per thread and TMA rings
// (kernels_aniso4.cu), tile width kAniso4TX, nz % 4 == 0, FP32 state
constexpr int kAniso4TX = 16;
struct Grad4Maps {
  CUtensorMap w1, m[4];  // w1 box (40, tx + 8); eps, del, pjx, pjy boxes (32, tx)
};
struct Div4Maps {
  CUtensorMap py, px, pz, w0, vel, w1;  // py (32, tx); px (32, tx + 8); pz (40, tx); w0 / vel / w1 (32, tx)
  // visco-acoustic update with its operands in the ring (qring 1: FP32 Q
  // memory, 2: BF16; 0: loaded by the update itself): the d0 / d1 halves
  // (box (32, tx, 1, order)) and 1/Q (box (32, tx))
  CUtensorMap qa, qb, iq;
  int qring;
};
// orders of the Q memory the divergence ring carries
constexpr int kDiv4QMax = 4;
bool aniso4_init();         // shared-memory attributes (call outside any capture)
int aniso4_ctas_per_sm();   // resident CTAs per SM of the interior divergence kernel
void launch_grad4(const GradArgs &a, const Tile4 *tiles, int ntiles, bool edge, int model, const Grad4Maps &m,
                  int *err, cudaStream_t st);
void launch_div4(const DivArgs &a, const Tile4 *tiles, int ntiles, bool edge, int mode, const Div4Maps &m, int *err,
                 cudaStream_t st);

// shot illumination compensation: optional box smoothing (half widths hxy, hz),
// damping factor from the mean (dsum: one double of scratch), image *= factor;
// tmp: one volume of scratch
void launch_illum_compensate(float *illum, float *tmp, float *image, double *dsum, int nx, int ny, int nz, int smooth,
                             int hxy, int hz, float amp_damping, float damp_weight, cudaStream_t st);

// INVERSION imaging condition (kernels_ic.cu): cuFFT plans, spectrum size in
// floats, and one imaging term of source slot io.src against receiver field u
// (S, Rv, Ds, Dr: volumes; Sh, Rh, Th: spectra); 0 or -1 (cuFFT failure)
void *ic_plans_create(int nx, int ny, int nz);
void ic_plans_destroy(void *plans);
long long ic_spectrum_floats(int nx, int ny, int nz);
int launch_ic_inversion(void *plans, const FusedIo &io, const float *u, float *S, float *Rv, float *Ds, float *Dr,
                        float *Sh, float *Rh, float *Th, int nx, int ny, int nz, float dx, float dy, float dz,
                        cudaStream_t st);

// FP16 fallback of the high-energy blocks of a learned snapshot (ae.cu): the
// blocks whose scale exceeds tau x the largest, largest first, at most cap
void ae_fallback_store(const float *w, const float *scales, int nx, int ny, int nz, float tau, long long cap, void *fb,
                       cudaStream_t st);
void ae_fallback_apply(const float *scales, int nx, int ny, int nz, long long cap, const void *fb, float *w,
                       cudaStream_t st);
size_t ae_fallback_bytes(long long cap);

// ---- compact FD (kernels_cfd.cu) -------------------------------------------
struct CfdPlanDev {
  int n;
  const float *bu, *bl, *am;  // [n][4] upper factor (super-diagonals 1..4), [n][4] multipliers, [60] A
  const float *rdiag;         // [n] 1 / pivot, from the FP64 factorisation
  const float *lm;            // [n][4] multipliers acting on row i: l[i-1][0], l[i-2][1], l[i-3][2], l[i-4][3]
  // rows [c0, c1] hold bitwise-identical (lm, bu, rdiag): the factors of the
  // Toeplitz interior have converged in FP32; c0 > c1 when there is no such run
  int c0, c1;
  float lmc[4], buc[4], rdc;
  float a[60];  // copy of am, read from the kernel-parameter (constant) bank
  // segment-parallel solve: nseg segments of seglen rows (the last one takes
  // the remainder, >= 8 rows); [n][4] tables: hf = response of the forward
  // value of row i to unit entering forward states of its segment, gb = the
  // segment-local back substitution of hf, hb = response of the backward
  // value to unit entering backward states (zero where a segment has none)
  int nseg, seglen;
  const float *hf, *gb, *hb;
};
// one-time attribute set-up of the compact-FD kernels (outside any capture)
int cfd_init();
// TMA box of the x / y line kernels: nb boxes of R rows (R <= 256) per tile
void cfd_tma_box(int n, int *R, int *nb);
// raw derivative of `in` along axis (0 x, 1 y, 2 z) into `out` (no PML).  For
// x / y, tensor maps of in / out with box (32, R, 1) / (32, 1, R) select the
// TMA tile kernel (null: plain loads and stores); err receives wait timeouts.
void launch_cfd_deriv(int axis, const CfdPlanDev &p, const float *in, float *out, int nx, int ny, int nz,
                      const CUtensorMap *tin, const CUtensorMap *tout, int *err, cudaStream_t st);
// x / y derivative by the register-streamed kernel (no shared memory)
// pipelined persistent x / y line solves over TMA tiles (one CTA per SM, a
// ring of tile buffers, right-hand side fused into the forward pass); false
// when a ring of three tiles does not fit in shared memory (nothing launched)
bool launch_cfd_deriv_pipe(int axis, const CfdPlanDev &p, int nx, int ny, int nz, const CUtensorMap *tin,
                           const CUtensorMap *tout, int *err, cudaStream_t st);
void launch_cfd_deriv_stream(int axis, const CfdPlanDev &p, const float *in, float *out, int nx, int ny, int nz,
                             cudaStream_t st);

// ---- segment-parallel compact-FD step (engine CFD, 3-D grids) --------------
// Five launches per step:
//   Z(w1) -> gz, X(w1) -> gx                     first derivatives, PML round 1
//   Y fused: Y(w1) -> gy, PML round 1; rho division and VTI / TTI scaling of
//            (gx, gy, gz) -> px, pz in place, py kept in shared memory;
//            Y(py) -> dy with PML round 2
//   Z(pz) -> dz                                  PML round 2
//   X fused: X(px) -> dx with PML round 2; w0 - vel (dx + dz + dy) (x, z, y in
//            turn, KernelCPU::TTI's order), then update2nd / the Q update
struct CfdSegArgs {
  int nx, ny, nz, pml3d, model, mode;
  PmlDev pml;
  QDev q;
  const float *w1, *vel, *eps, *del, *pjx, *pjy, *rho;  // rho null: no density model
  float *w0;
  float *gx, *gz;  // x / z gradients, overwritten by the scaled px / pz
  float *dz, *dy;  // divergence parts along z and y
};
int cfd_seg_init();
// largest line length the segment-parallel kernels take along axis (shared memory)
int cfd_seg_max_n(int axis);
// Z or X line derivative of `in` into `out`, PML round `round` on that component;
// tin: tensor map of `in` with box (32, R, 1) for X (null: plain loads)
void launch_cfd_seg_line(int axis, int round, const CfdPlanDev &p, const float *in, float *out, const CfdSegArgs &a,
                         const CUtensorMap *tin, int *err, cudaStream_t st);
// the fused y kernel (plans pg: gradient pass, pd: divergence pass; tin: map of
// w1 with box (32, 1, R)) and the fused x kernel (tin: map of px, box (32, R, 1))
void launch_cfd_seg_yfused(const CfdPlanDev &pg, const CfdPlanDev &pd, const CfdSegArgs &a, const CUtensorMap *tin,
                           int *err, cudaStream_t st);
void launch_cfd_seg_xfused(const CfdPlanDev &p, const CfdSegArgs &a, const CUtensorMap *tin, int *err,
                           cudaStream_t st);

struct CfdGradEpiArgs {  // PML round 1 + scaling on raw gradients, in place
  int nx, ny, nz, pml3d, model;
  float *gx, *gy, *gz;
  const float *eps, *del, *pjx, *pjy;
  const float *rho;  // density (null: none): the gradient is divided by it
  PmlDev pml;
  FusedIo io;
  const float *w1;
};
void launch_cfd_grad_epilogue(const CfdGradEpiArgs &a, cudaStream_t st, bool pml_only = false);

struct CfdDivEpiArgs {  // PML round 2 on raw divergence parts + update
  int nx, ny, nz, pml3d, mode;
  const float *dx, *dy, *dz;
  const float *w1;
  float *w0;
  const float *vel;
  // density (null: none) and the engine's form of the accumulation with it:
  // 0 FdEngine_cfd, 1 FdEngine_r2c / _r2r, 2 the Derivative path
  const float *rho;
  int rho_form;
  PmlDev pml;
  QDev q;
};
void launch_cfd_div_epilogue(const CfdDivEpiArgs &a, cudaStream_t st, bool pml_only = false);
// the z line solve of `in` fused with the gradient / divergence epilogue (the
// raw z part stays in shared memory; the x / y parts come from a.gx, a.gy /
// a.dx, a.dy)
void launch_cfd_zgrad(const CfdPlanDev &p, const float *in, const CfdGradEpiArgs &a, cudaStream_t st);
void launch_cfd_zdiv(const CfdPlanDev &p, const float *in, const CfdDivEpiArgs &a, cudaStream_t st);  // mode 0 / 1

// ---- double-grid IMAGE1 imaging condition (kernels_ic.cu) -------------------
// dz / dx / dy: 1 or 2 per axis; iv[k]: the copy holding the z, x, y, zx, zy,
// xy, zxy half shift (0: not made; ImagingCorrelator's ivz .. ivzxy); nloop
// copies (1, 2, 4 or 8); slot[c]: the copy on doubled-grid points of class
// c = 4 (y odd) + 2 (x odd) + (z odd)
struct DblMap {
  int dz, dx, dy, nloop;
  int iv[7];
  int slot[8];
};
struct FftPlans;
// one imaging step: S[0..nloop) / Rv[0..nloop) scratch volumes, image / comp
// nloop cubes each, illum (null: off) on the base grid
int launch_ic_double(FftPlans *fft, const DblMap &m, const FusedIo &io, const float *u, float *const *S,
                     float *const *Rv, float *image, float *comp, float *illum, int nx, int ny, int nz, float high_z,
                     float high_xy, cudaStream_t st);
void launch_dbl_interleave(const float *cubes, float *out, const DblMap &m, int nx, int ny, int nz, cudaStream_t st);
void launch_dbl_illum(const float *in, float *out, const DblMap &m, int nx, int ny, int nz, cudaStream_t st);
// kind 0: half shift to x + d/2; kind 1: high cut above `high` of Nyquist (in may equal out)
int launch_fft_filter(FftPlans *p, int axis, int kind, float high, const float *in, float *out, cudaStream_t st);

// ---- pseudo-spectral first derivative, FFTWR2C engine (kernels_fft.cu) -------
struct FftPlans;
// cuFFT plans of the three axes (y skipped when ny == 1) bound to stream st,
// the wavenumber tables and the spectrum / transpose scratch
// tensor_cores: the derivatives as circulant line matrices by the split-TF32
// tcgen05 kernel where it applies (nz % 4 == 0, lines of at most 512 points);
// err: device flag its bounded waits raise
int fft_plans_create(FftPlans **out, int nx, int ny, int nz, float dx, float dy, float dz, cudaStream_t st,
                     bool tensor_cores = false, int *err = nullptr);
void fft_plans_destroy(FftPlans *p);
// raw derivative of `in` along axis (0 x, 1 y, 2 z) into `out` (no PML);
// isign +1 / -1 as FdEngine_r2c::fftderiv1_r2c's (the sign of bin n/2 for odd n)
int launch_fft_deriv(FftPlans *p, int axis, int isign, const float *in, float *out, cudaStream_t st);
// FFTWR2R engine: one line matrix per axis and pass, applied as FP32 GEMMs on
// stream st (cuBLAS handle, fixed workspace)
struct R2rPlans;
// tensor_cores: the line operators by the split-TF32 tcgen05 kernel where it
// applies (nz % 4 == 0, lines of at most 512 points); err: device flag its
// bounded waits raise
int r2r_plans_create(R2rPlans **out, int nx, int ny, int nz, float dx, float dy, float dz, cudaStream_t st,
                     bool tensor_cores, int *err);
// tcgen05 z-line operator (kernels_r2r_tc.cu)
size_t r2r_tc_smem(int n);
bool r2r_tc_supported(int axis, int nx, int ny, int nz);
size_t r2r_tc_bytes(int n);  // the pre-arranged TF32 parts of one n x n line matrix
int r2r_tc_init();
void launch_tf32_arrange(const float *D, unsigned char *Bg, int n, cudaStream_t st);
void launch_r2r_tc(int axis, const float *in, float *out, const unsigned char *Bg, int nx, int ny, int nz, int *err,
                   cudaStream_t st);
void r2r_plans_destroy(R2rPlans *p);
int launch_r2r_deriv(R2rPlans *p, int axis, int isign, const float *in, float *out);

// ---- wavefield I/O, sources, receivers, snapshots (kernels_io.cu) -----------
void launch_update2nd(float *w0, const float *w1, const QDev *q, long long n, cudaStream_t st);
// atomic scatter of every trace of `t` (Receiver::apply_src)
void launch_inject_scatter(const TraceDev &t, int it, float *w0, const float *vel, int nx, int ny, int nz,
                           cudaStream_t st);
// grouped injection: xy plane gather then z expansion
void launch_inject_group(const GroupDev &gr, const TraceDev &t, int it, float *plane, float *w0, const float *vel,
                         int nx, int ny, int nz, cudaStream_t st);
void launch_extract_direct(const TraceDev &t, const float *w0, float *out, int jt, int nt_out, int nx, int ny, int nz,
                           cudaStream_t st);
void launch_extract_group(const GroupDev &gr, const TraceDev &t, const float *w0, float *plane, float *out, int jt,
                          int nt_out, int nx, int ny, int nz, cudaStream_t st);
// per-y-slab max |w| -> slab[iy]; c16 header written into hdr (may be null)
void launch_slab_max(const float *w, float *slab, uint16_t *c16_base, int fmt, int nx, int ny, int nz, cudaStream_t st);
// standalone snapshot store / IC (same arithmetic as the fused path)
void launch_fused_io(const FusedIo &io, const float *u, int nx, int ny, int nz, cudaStream_t st);
// decode a snapshot slot (with decode tapers when ex/ey/ez given)
void launch_snap_decode(const SnapDev &s, float *out, const float *ex, const float *ey, const float *ez, int nx, int ny,
                        int nz, cudaStream_t st);
// COMPRESS_16 on device buffers
void launch_c16_compress(const float *in, uint16_t *out, float *slab, int nx, int ny, int nz, cudaStream_t st);
void launch_c16_uncompress(const uint16_t *in, float *out, float *slab, const float *ex, const float *ey,
                           const float *ez, int nx, int ny, int nz, cudaStream_t st);
void launch_vel2(float *vel, float *invq, long long n, float dt2, float cq0, int use_q, cudaStream_t st);
// NaN/Inf scan: sets *flag = 1 when any value is not finite
void launch_nonfinite_scan(const float *w, long long n, int *flag, cudaStream_t st);

// ---- learned snapshot compressor (ae.cu) --------------------------------------
long long ae_volume_blocks(int nx, int ny, int nz);  // 8^3 blocks covering a volume
int ae_prepare(rtm_ae *a);                           // workspace (call outside any capture)
// volume -> latents [nb][32] + scales [nb]; latents + scales -> volume (device, stream st)
int ae_compress(rtm_ae *a, const float *w, int nx, int ny, int nz, void *latent, float *scales, cudaStream_t st);
int ae_decompress(rtm_ae *a, const void *latent, const float *scales, int nx, int ny, int nz, float *w,
                  cudaStream_t st);

}  // namespace rtm
