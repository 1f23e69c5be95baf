// rtm_capi.cu - the engine behind include/rtm_b200.h: device state of one shot,
// the time-loop drivers (Propagator::modelling / migration) captured as CUDA
// graphs, and every extern "C" entry point.  No entry point throws or aborts;
// CUDA failures become RTM_ERR_CUDA with the message kept on the handle.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <array>
#include <vector>

#include <cuda.h>

#include "../../include/rtm_b200.h"
#include "host_setup.h"
#include "kernel_api.h"

namespace rtm {

static std::string g_create_error;

struct TraceSetDev {
  int ntr = 0, lx = 0, ly = 0, lz = 0, nt = 0;
  float scaler = 1.f;
  int *off = nullptr, *len = nullptr;
  float *kx = nullptr, *ky = nullptr, *kz = nullptr, *traces = nullptr;
  float *out = nullptr;  // extraction results [ntr][nt]
  int *ungrouped = nullptr;
  int n_ungrouped = 0;
  std::vector<GroupDev> groups;
  std::vector<void *> group_allocs;
  TraceDev dev() const {
    TraceDev t{};
    t.ntr = ntr, t.lx = lx, t.ly = ly, t.lz = lz, t.nt = nt;
    t.off = off, t.len = len, t.kx = kx, t.ky = ky, t.kz = kz, t.traces = traces, t.scaler = scaler;
    return t;
  }
};

// A device table of 32 (z) x tx (x) column tiles over y segments of yseg
// planes: n_int tiles free of PML cells, then n_edge tiles that may hold some.
struct TileSet {
  Tile4 *d = nullptr;
  int cap = 0, n_int = 0, n_edge = 0, tx = 0, yseg = 0;
  bool current(int tx_, int yseg_) const { return d && tx == tx_ && yseg == std::max(1, yseg_); }
};

struct Engine {
  rtm_dims d{};
  rtm_config c{};
  // FD8 ISO without density: the Laplacian path (KernelCPU::ISO, do_laplacian);
  // every other configuration takes the two first-derivative passes
  // (bgprtm/KernelCPU.cpp:125-174)
  bool lap_iso() const { return c.engine == RTM_ENGINE_FD8 && c.model_type == RTM_ISO && !c.use_rho; }
  int device = 0;
  cudaStream_t st = nullptr;
  long long n = 0, nxz = 0;
  std::string err;
  std::vector<void *> allocs;
  // state
  float *w0 = nullptr, *w1 = nullptr, *vel = nullptr;
  float *eps = nullptr, *del = nullptr, *pjx = nullptr, *pjy = nullptr, *invq = nullptr;
  float *rho = nullptr;  // density (KernelCPU::setModel's rho), null without a density model
  float *wq[2] = {nullptr, nullptr};
  int iq0 = 0;
  float *px = nullptr, *py = nullptr, *pz = nullptr;  // gradient scratch (anisotropic / CFD)
  float *scr = nullptr, *scr2 = nullptr;              // CFD raw-derivative scratch
  float c1x[5], c1y[5], c1z[5], c2x[5], c2y[5], c2z[5];
  CfdPlanDev cfd[3][2] = {};
  FftPlans *fft = nullptr;   // FFTWR2C engine: cuFFT plans and scratch
  R2rPlans *r2r = nullptr;   // FFTWR2R engine: line matrices and the GEMM handle
  int fft_err = 0;           // a cuFFT execution failed
  PmlDev pml{};
  int model_set = 0;
  // Q
  float cq0 = 0.f, cqsum = 0.f, cq[8] = {}, cwq[8] = {};
  int q_set = 0;
  // traces
  TraceSetDev inj, ext;
  float *plane = nullptr;
  // snapshots
  int snap_fmt = 0, nslots = 0;
  size_t slot_bytes = 0;
  char *snaps = nullptr;
  // snapshot offload (rtm_snapshot_offload): the slots live in pinned host memory and
  // `nstage` device slots (snaps) stage them; slot s uses staging slot s % nstage.
  // Copies run on st_copy, forked from st by events and joined back before every
  // graph capture ends; stage_ev[k] marks the last copy into / out of staging slot k.
  float *illum = nullptr;  // source illumination (rtm_illum_setup), accumulated by the imaging condition
  int illum_on = 0;
  // imaging condition (rtm_image_condition): 0 zero-lag correlation fused into the
  // step, 1 INVERSION with cuFFT derivatives (plans and scratch volumes / spectra)
  int ic_opt = 0;
  void *ic_plans = nullptr;
  float *icS = nullptr, *icR = nullptr, *icDs = nullptr, *icDr = nullptr, *icSh = nullptr, *icRh = nullptr,
        *icTh = nullptr;
  // double-grid IMAGE1 (rtm_image_double): copy map, filters, line-FFT plans,
  // the fields' nloop copies and the nloop image cubes (+ compensation)
  int dbl = 0;
  DblMap dmap{};
  float dbl_hz = 0.9f, dbl_hxy = 0.7f;
  FftPlans *dbl_fft = nullptr;
  float *dblS[8] = {}, *dblR[8] = {};
  float *dbl_img = nullptr, *dbl_comp = nullptr;
  char *host_snaps = nullptr;
  int nstage = 0;
  cudaStream_t st_copy = nullptr;
  cudaEvent_t ev_fork = nullptr, stage_ev[8] = {};
  int stage_slot[8] = {};  // slot a staging buffer holds (-1: none)
  bool stage_wait[8] = {};  // st has not yet waited for the last copy into / out of it
  float *slabs = nullptr;  // [nslots][ny]
  std::vector<char> stored;
  // imaging
  float *image = nullptr, *comp = nullptr;
  float *ex = nullptr, *ey = nullptr, *ez = nullptr, *one_x = nullptr, *one_y = nullptr, *one_z = nullptr;
  float *taper_z = nullptr;
  std::vector<float> taper_t;
  int ic_edge = 1;
  // launch shape and timing
  int tx = 8, yseg = 16;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  int *dflag = nullptr;
  int *nfflag = nullptr;  // result of the non-finite scan (allocated on first use)
  rtm_ae *ae = nullptr;      // learned compressor of RTM_SNAP_AE snapshots
  float ae_fb_tau = 0.f;     // FP16 fallback of learned snapshots: blocks above tau x the largest scale,
  float ae_fb_frac = 0.f;    // at most this fraction of the blocks (0: no fallback)
  // FP16 wavefield state (state_fp16): h0 / h1 play w0 / w1, value = half * s[iy];
  // sn is the scale of the field the current step writes; m0 / m1 slab maxima
  int f16 = 0;
  __half *h0 = nullptr, *h1 = nullptr;
  float *s0 = nullptr, *s1 = nullptr, *sn = nullptr;
  unsigned *m0 = nullptr, *m1 = nullptr;
  float f16_floor = 1e-20f;  // smallest slab max a scale is built for (source amplitude)
  float vel2max = 0.f;       // max (v dt)^2 of the model
  float *ae_scratch = nullptr;  // decoded source snapshot for the imaging condition
  // launch accounting and the optional per-kernel event profile
  long long launches = 0;
  int use_tma = 0;
  // ISO FD8 with 4 z cells per thread (takes precedence over use_tma): 0 off,
  // 1 register-prefetch kernel (tile width v4_tx), 2 TMA rings (kIso4TmaShapes[v4_shape])
  int iso4 = 0;
  int v4_tx = 16, v4_shape = 0, v4_yseg = 16;
  // column-tile tables (interior tiles [0, n_int), then PML tiles) of the
  // ISO TMA-ring kernel and of the FD8 gradient / divergence passes
  TileSet t_iso, t_fd8;
  // FD8 VTI / TTI with 4 z cells per thread and TMA rings (kernels_aniso4.cu) and its y segment
  int aniso4 = 0, an4_yseg = 16;
  TileSet t_an4;
  std::vector<std::array<int, 4>> tune_desc;  // candidates of the last rtm_autotune and their times
  std::vector<float> tune_ms;
  int cfd_tma = 0;  // tensor maps of the volume can be made (nz % 4 == 0)
  int cfd_xy = 0;   // compact-FD x / y kernel: 0 streamed, 1 TMA tile, 2 plain tile (the split
                    // pipeline: line solves + pointwise epilogues); 3 / 4 the segment-parallel
                    // fused pipeline with TMA / plain tile loads
  int cfd_seg_ok = 0;  // the segment-parallel pipeline applies (engine CFD, 3-D, lines fit)
  int cfd_zfuse = 0;   // the z line solves carry the interior box of the epilogues (kernel_variant 9)
  int cfd_pipe = 0;    // x / y line solves by the pipelined persistent TMA kernel (kernel_variant 10)
  int tma_shape = 1;  // index into kIsoTmaShapes
  struct TMap {
    const void *p;
    int bz, bx, by;
    CUtensorMap m;
  };
  std::vector<TMap> tmaps;
  // checkpoints of the propagation state (rtm_checkpoint_setup): nckpt slots of
  // ckpt_bytes; the loops map step it to snapshot slot it / interval - slot0
  char *ckpts = nullptr;
  int nckpt = 0;
  size_t ckpt_bytes = 0;
  int slot0 = 0;
  int qring_ok = 1;  // the divergence ring may carry the Q memory (not kernel_variant 7)
  int prof_on = 0;
  struct ProfRec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof_recs;
  double prof_ms[RTM_NKINDS] = {};
  long long prof_cnt[RTM_NKINDS] = {};

  template <typename T> int alloc(T *&p, size_t count) {
    void *v = nullptr;
    cudaError_t e = cudaMalloc(&v, count * sizeof(T));
    if (e != cudaSuccess) {
      err = std::string("cudaMalloc(") + std::to_string(count * sizeof(T)) + " bytes): " + cudaGetErrorString(e);
      cudaGetLastError();
      return RTM_ERR_NOMEM;
    }
    allocs.push_back(v);
    p = (T *)v;
    return RTM_OK;
  }
  void release(void *p) {
    if (!p) return;
    auto it = std::find(allocs.begin(), allocs.end(), p);
    if (it != allocs.end()) allocs.erase(it);
    cudaFree(p);
  }
};

int cuda_fail(cudaError_t e, const char *what, Engine *h) {
  if (h) h->err = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? RTM_ERR_NOMEM : RTM_ERR_CUDA;
}

#define CK(call) RTM_CUDA_OK(call)
#define TRY(expr)                 \
  do {                            \
    int r__ = (expr);             \
    if (r__ != RTM_OK) return r__; \
  } while (0)

static int check_launch(Engine *h, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what, h);
  if (h->fft_err) {
    h->fft_err = 0;
    h->err = std::string(what) + ": cuFFT / cuBLAS execution failed";
    return RTM_ERR_CUDA;
  }
  return RTM_OK;
}

// a bounded device wait that gave up raises the engine's flag
static int check_flag(Engine *h) {
  int f = 0;
  CK(cudaMemcpy(&f, h->dflag, sizeof f, cudaMemcpyDeviceToHost));
  if (f) {
    cudaMemset(h->dflag, 0, sizeof f);
    h->err = "a pipelined kernel's bounded wait for its tile copies gave up";
    return RTM_ERR_TIMEOUT;
  }
  return RTM_OK;
}

// Counts one kernel launch of `kind`; when profiling, brackets it with events.
struct KScope {
  Engine *h;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  KScope(Engine *h_, int k, int n = 1) : h(h_), kind(k) {
    h->launches += n;
    if (h->prof_on) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, h->st);
    }
  }
  ~KScope() {
    if (h->prof_on) {
      cudaEventRecord(b, h->st);
      h->prof_recs.push_back({kind, a, b});
    }
  }
};

static void prof_collect(Engine *h) {
  for (auto &r : h->prof_recs) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      h->prof_ms[r.kind] += ms;
      h->prof_cnt[r.kind] += 1;
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  h->prof_recs.clear();
  cudaGetLastError();
}

// launch shape: 32 x tx column tiles, y split so the grid covers the 148 SMs
static void choose_shape(Engine *h) {
  const int nx = h->d.nx, ny = h->d.ny, nz = h->d.nz;
  int tx = 8;
  long long bxz = (long long)((nz + 31) / 32) * ((nx + tx - 1) / tx);
  long long want = 148LL * 2 * 8;  // ~8 waves of 2 CTAs per SM
  int nseg = (int)std::max(1LL, std::min<long long>((want + bxz - 1) / bxz, std::max(1, ny / 16)));
  h->tx = tx;
  h->yseg = (ny + nseg - 1) / nseg;
}

// y segment length for a tile width: enough CTAs for ~8 waves of 2 per SM
static int yseg_for(Engine *h, int tx) {
  const int nx = h->d.nx, ny = h->d.ny, nz = h->d.nz;
  long long bxz = (long long)((nz + 31) / 32) * ((nx + tx - 1) / tx);
  long long want = 148LL * 2 * 8;
  int nseg = (int)std::max(1LL, std::min<long long>((want + bxz - 1) / bxz, std::max(1, ny / 16)));
  return (ny + nseg - 1) / nseg;
}

// y segment of the 4-z-cell ISO kernel at tile width tx: the count of
// segments whose waves of resident CTAs cover the y planes in the fewest
// plane-steps (a segment re-reads an 8-plane y halo, mostly from L2)
static int yseg_v4(Engine *h, int tx, int ctas_per_sm) {
  const int nx = h->d.nx, ny = h->d.ny, nz = h->d.nz;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const long long bxz = (long long)((nz + 31) / 32) * ((nx + tx - 1) / tx);
  const long long res = (long long)std::max(1, nsm) * std::max(1, ctas_per_sm);
  int best_y = ny;
  double best = 1e300;
  for (int nseg = 1; nseg <= std::max(1, ny / 8); nseg++) {
    const int yseg = (ny + nseg - 1) / nseg;
    const long long ctas = bxz * ((ny + yseg - 1) / yseg);
    const double cost = (double)((ctas + res - 1) / res) * (yseg + 3);
    if (cost < best * 0.98) best = cost, best_y = yseg;
  }
  return best_y;
}
// Tile table for tile width tx and y segment yseg: columns touching an x or
// z PML face are PML tiles over all y; the others are PML tiles over the y
// faces and interior tiles between.  Built on the host and uploaded (never
// inside a stream capture).
static int build_tiles(Engine *h, TileSet &t, int tx, int yseg) {
  yseg = std::max(1, yseg);
  if (t.current(tx, yseg)) return RTM_OK;
  const int nx = h->d.nx, ny = h->d.ny, nz = h->d.nz;
  const int zl = h->pml.f[DZ][0].w, zh = h->pml.f[DZ][1].w, xl = h->pml.f[DX][0].w, xh = h->pml.f[DX][1].w,
            yl = h->pml.f[DY][0].w, yh = h->pml.f[DY][1].w;
  std::vector<Tile4> in, ed;
  auto segs = [&](std::vector<Tile4> &v, int bz, int bx, int a, int b) {
    for (int y = a; y < b; y += yseg) v.push_back({bz, bx, y, std::min(b, y + yseg)});
  };
  const int nbz = (nz + 31) / 32, nbx = (nx + tx - 1) / tx;
  for (int bx = 0; bx < nbx; bx++)
    for (int bz = 0; bz < nbz; bz++) {
      const bool exz = bx * tx < xl || std::min(nx, (bx + 1) * tx) > nx - xh || bz * 32 < zl ||
                       std::min(nz, bz * 32 + 32) > nz - zh;
      if (exz) {
        segs(ed, bz, bx, 0, ny);
      } else {
        segs(ed, bz, bx, 0, yl);
        segs(in, bz, bx, yl, ny - yh);
        segs(ed, bz, bx, ny - yh, ny);
      }
    }
  // launch order: y segment slowest, then x, then z (neighbouring CTAs share halos)
  auto by_y = [](const Tile4 &a, const Tile4 &b) {
    return a.y0 != b.y0 ? a.y0 < b.y0 : a.bx != b.bx ? a.bx < b.bx : a.bz < b.bz;
  };
  std::stable_sort(in.begin(), in.end(), by_y);
  std::stable_sort(ed.begin(), ed.end(), by_y);
  const int n = (int)(in.size() + ed.size());
  if (n > t.cap) {
    h->release(t.d);
    t.d = nullptr, t.cap = 0;
    TRY(h->alloc(t.d, (size_t)n));
    t.cap = n;
  }
  std::vector<Tile4> all(in);
  all.insert(all.end(), ed.begin(), ed.end());
  CK(cudaMemcpy(t.d, all.data(), sizeof(Tile4) * n, cudaMemcpyHostToDevice));
  t.n_int = (int)in.size(), t.n_edge = (int)ed.size(), t.tx = tx, t.yseg = yseg;
  return RTM_OK;
}
static int iso4_tiles(Engine *h) {
  return build_tiles(h, h->t_iso, kIso4TmaShapes[h->v4_shape].tx, h->v4_yseg);
}
// tables of the FD8 gradient / divergence passes (tile width tx, y segment yseg)
static int fd8_tiles(Engine *h) { return build_tiles(h, h->t_fd8, h->tx, h->yseg); }
static int an4_tiles(Engine *h) { return build_tiles(h, h->t_an4, kAniso4TX, h->an4_yseg); }

static int yseg_an4(Engine *h) { return yseg_v4(h, kAniso4TX, aniso4_ctas_per_sm()); }

static int yseg_iso4(Engine *h) {
  if (h->iso4 == 2)
    return yseg_v4(h, kIso4TmaShapes[h->v4_shape].tx, iso_tma4_ctas_per_sm(h->v4_shape, h->c.pml3d));
  return yseg_v4(h, h->v4_tx, iso_v4_ctas_per_sm(h->v4_tx, h->c.pml3d));
}

// Segment layout of the segment-parallel solve of an n-point line (segments
// of seglen rows, a multiple of 8, at most 8 of them, the last one >= 8 rows)
// and its correction tables [n][4] (see kernels_cfd.cu): hf = forward
// responses to unit entering states y_{b-1-k}, gb = their segment-local back
// substitutions, hb = backward responses to unit entering states f_{e+k}.
// FP64 recurrences on the FP32 factors the kernels use.
static void cfd_seg_layout(int n, int &nseg, int &seglen) {
  seglen = ((n + 7) / 8 + 7) / 8 * 8;
  nseg = (n + seglen - 1) / seglen;
  if (nseg > 1 && n - (nseg - 1) * seglen < 8) nseg--;
}
static void cfd_seg_tables(int n, const std::vector<float> &lm, const std::vector<float> &bu,
                           const std::vector<float> &rd, int nseg, int seglen, std::vector<float> &hf,
                           std::vector<float> &gb, std::vector<float> &hb) {
  hf.assign(4 * (size_t)n, 0.f), gb.assign(4 * (size_t)n, 0.f), hb.assign(4 * (size_t)n, 0.f);
  // back substitution of y over rows [b, e) with f_{e..e+3} given in f[e-b ..]
  auto back = [&](int b, int e, const std::vector<double> &y, std::vector<double> &f) {
    for (int i = e - 1; i >= b; i--) {
      const float *u = &bu[4 * (size_t)i];
      double w = y[i - b];
      for (int k = 3; k >= 0; k--) w -= (double)u[k] * f[i - b + 1 + k];
      f[i - b] = w * (double)rd[i];
    }
  };
  for (int j = 0; j < nseg; j++) {
    const int b = j * seglen, e = j == nseg - 1 ? n : b + seglen, len = e - b;
    for (int k = 0; k < 4; k++) {
      if (j > 0) {
        std::vector<double> y(len + 4, 0.0);  // y[4 + i - b] = y_i; y[3 - q] = y_{b-1-q}
        y[3 - k] = 1.0;
        for (int i = b; i < e; i++) {
          const float *m = &lm[4 * (size_t)i];  // multipliers of y_{i-1} .. y_{i-4}
          double v = 0.0;
          for (int q = 3; q >= 0; q--) v -= (double)m[q] * y[4 + i - b - 1 - q];
          y[4 + i - b] = v;
          hf[4 * (size_t)i + k] = (float)v;
        }
        std::vector<double> yi(y.begin() + 4, y.end()), f(len + 4, 0.0);
        back(b, e, yi, f);
        for (int i = b; i < e; i++) gb[4 * (size_t)i + k] = (float)f[i - b];
      }
      if (j < nseg - 1) {
        std::vector<double> y(len, 0.0), f(len + 4, 0.0);
        f[len + k] = 1.0;
        back(b, e, y, f);
        for (int i = b; i < e; i++) hb[4 * (size_t)i + k] = (float)f[i - b];
      }
    }
  }
}

// Longest run of rows whose (lm, bu, rdiag) are bitwise identical: in the
// interior of a line the LU of the Toeplitz band matrix has converged, and
// the line kernels hold those factors in registers instead of loading them.
static void cfd_constant_run(int n, const std::vector<float> &lm, const std::vector<float> &bu,
                             const std::vector<float> &rd, CfdPlanDev &pd) {
  auto same = [&](int i, int j) {
    return !memcmp(&lm[(size_t)i * 4], &lm[(size_t)j * 4], 16) && !memcmp(&bu[(size_t)i * 4], &bu[(size_t)j * 4], 16) &&
           !memcmp(&rd[i], &rd[j], 4);
  };
  int best = 0, blo = 0;
  for (int lo = 0; lo < n;) {
    int hi = lo;
    while (hi + 1 < n && same(lo, hi + 1)) hi++;
    if (hi - lo + 1 > best) best = hi - lo + 1, blo = lo;
    lo = hi + 1;
  }
  if (best < 16) {
    pd.c0 = 1, pd.c1 = 0;
    return;
  }
  pd.c0 = blo, pd.c1 = blo + best - 1;
  for (int k = 0; k < 4; k++) pd.lmc[k] = lm[(size_t)blo * 4 + k], pd.buc[k] = bu[(size_t)blo * 4 + k];
  pd.rdc = rd[blo];
}

static PmlDev pml_dev(Engine *h) { return h->pml; }

// tensor map of the Q memory half at p ([order][ny][nx][nz], FP32 or BF16)
// with box (32, bx, 1, order), cached like tmap (by = -order marks the 4-D map)
static bool tmap_q(Engine *h, const void *p, int bx, CUtensorMap *out) {
  const int L = h->c.q_order;
  for (const auto &t : h->tmaps)
    if (t.p == p && t.bz == 32 && t.bx == bx && t.by == -L) {
      *out = t.m;
      return true;
    }
  Engine::TMap t{p, 32, bx, -L, {}};
  if (!make_tmap_q(&t.m, p, h->d.nx, h->d.ny, h->d.nz, L, h->c.q_bf16 != 0, 32, bx)) return false;
  h->tmaps.push_back(t);
  *out = t.m;
  return true;
}

// tensor map of a device volume with box (bz, bx, 1), built once per buffer;
// returned by value (the cache may grow and move its entries)
static bool tmap(Engine *h, const void *p, int bz, int bx, CUtensorMap *out, int by = 1) {
  for (const auto &t : h->tmaps)
    if (t.p == p && t.bz == bz && t.bx == bx && t.by == by) {
      *out = t.m;
      return true;
    }
  Engine::TMap t{p, bz, bx, by, {}};
  if (!make_tmap(&t.m, p, h->d.nx, h->d.ny, h->d.nz, bz, bx, by)) return false;
  h->tmaps.push_back(t);
  *out = t.m;
  return true;
}

// one compact-FD line derivative.  x / y: the register-streamed kernel
// (cfd_xy 0), the TMA tile kernel (1, when the tensor maps can be made:
// nz % 4 == 0) or the plain staged tile kernel (2)
static void cfd_deriv(Engine *h, int axis, int sgn, const float *in, float *out) {
  const rtm_dims &d = h->d;
  // the Derivative path's divergence pass takes isign = iswitch: 1 for TTI,
  // 2 otherwise (bgprtm/Derivative.cpp:4-8, 92-112)
  const bool deriv_path = h->c.engine == RTM_ENGINE_CFDB || h->c.engine == RTM_ENGINE_FFTV ||
                          h->c.engine == RTM_ENGINE_SINCOS;
  if (sgn && deriv_path && h->c.model_type == RTM_TTI) sgn = 0;
  if (h->fft) {  // FFTWR2C: isign +1 in the gradient pass, -1 in the divergence pass; FFTV: +1 in both
    const int isign = h->c.engine == RTM_ENGINE_FFTV ? 1 : sgn ? -1 : 1;
    if (launch_fft_deriv(h->fft, axis, isign, in, out, h->st) != RTM_OK) h->fft_err = 1;
    return;
  }
  if (h->r2r) {  // FFTWR2R, the same pass signs; SINCOS: runCosSin for isign 1, runSinCos otherwise
    if (launch_r2r_deriv(h->r2r, axis, sgn ? -1 : 1, in, out) != RTM_OK) h->fft_err = 1;
    return;
  }
  // CFD_BATCH: the divergence-pass plan from iswitch (above): plan 1 for TTI
  if (axis != DZ && h->cfd_xy == 0) {
    launch_cfd_deriv_stream(axis, h->cfd[axis][sgn], in, out, d.nx, d.ny, d.nz, h->st);
    return;
  }
  CUtensorMap mi, mo;
  bool tma = false;
  if (axis != DZ && h->cfd_xy == 1 && h->cfd_tma) {
    int R, nb;
    cfd_tma_box(axis == DX ? d.nx : d.ny, &R, &nb);
    const int bx = axis == DX ? R : 1, by = axis == DX ? 1 : R;
    tma = tmap(h, in, 32, bx, &mi, by) && tmap(h, out, 32, bx, &mo, by);
  }
  if (tma && h->cfd_pipe &&
      launch_cfd_deriv_pipe(axis, h->cfd[axis][sgn], d.nx, d.ny, d.nz, &mi, &mo, h->dflag, h->st))
    return;
  launch_cfd_deriv(axis, h->cfd[axis][sgn], in, out, d.nx, d.ny, d.nz, tma ? &mi : nullptr, tma ? &mo : nullptr,
                   h->dflag, h->st);
}

static int setup_pml(Engine *h) {
  const rtm_config &c = h->c;
  const int nn[3] = {h->d.nx, h->d.ny, h->d.nz};
  const double dd[3] = {h->d.dx, h->d.dy, h->d.dz};
  const bool second = h->lap_iso();
  const int ncomp = (!c.pml3d || second) ? 1 : 3;
  for (int dim = 0; dim < 3; dim++)
    for (int s = 0; s < 2; s++) {
      PmlFace &F = h->pml.f[dim][s];
      F = PmlFace{};
      int w = c.nbnd[2 * dim + s];
      bool on = w > 1 && !(dim == DZ && s == SIDE_LO && !c.top_pml);
      if (!on) continue;
      if (w * 2 > nn[dim] && !(nn[dim] == 1)) {
        h->err = "PML wider than half the grid";
        return RTM_ERR_ARG;
      }
      std::vector<float> co;
      pml_profile(w, dd[dim], h->d.dt, c.vmax, c.pml_eps, c.pml3d_scaler, co);
      float *dco;
      TRY(h->alloc(dco, co.size()));
      CK(cudaMemcpy(dco, co.data(), co.size() * 4, cudaMemcpyHostToDevice));
      F.w = w;
      F.co = dco;
      long long plane = dim == DX ? (long long)h->d.ny * h->d.nz
                                  : dim == DY ? (long long)h->d.nx * h->d.nz : (long long)h->d.nx * h->d.ny;
      for (int r = 0; r < 2; r++)
        for (int k = 0; k < ncomp; k++) TRY(h->alloc(F.q[r][k], (size_t)plane * w));
    }
  return RTM_OK;
}

static int zero_state(Engine *h) {
  if (h->f16) {
    CK(cudaMemsetAsync(h->h0, 0, h->n * 2, h->st));
    CK(cudaMemsetAsync(h->h1, 0, h->n * 2, h->st));
    CK(cudaMemsetAsync(h->m0, 0, h->d.ny * 4, h->st));
    CK(cudaMemsetAsync(h->m1, 0, h->d.ny * 4, h->st));
    launch_f16_scales(h->m0, h->m1, h->s0, h->d.ny, h->f16_floor, h->st);
    launch_f16_scales(h->m0, h->m1, h->s1, h->d.ny, h->f16_floor, h->st);
    launch_f16_scales(h->m0, h->m1, h->sn, h->d.ny, h->f16_floor, h->st);
  } else {
    CK(cudaMemsetAsync(h->w0, 0, h->n * 4, h->st));
    CK(cudaMemsetAsync(h->w1, 0, h->n * 4, h->st));
  }
  for (int dim = 0; dim < 3; dim++)
    for (int s = 0; s < 2; s++) {
      PmlFace &F = h->pml.f[dim][s];
      if (!F.w) continue;
      long long plane = dim == DX ? (long long)h->d.ny * h->d.nz
                                  : dim == DY ? (long long)h->d.nx * h->d.nz : (long long)h->d.nx * h->d.ny;
      for (int r = 0; r < 2; r++)
        for (int k = 0; k < 3; k++)
          if (F.q[r][k]) CK(cudaMemsetAsync(F.q[r][k], 0, plane * F.w * 4, h->st));
    }
  if (h->c.use_q && h->wq[0]) {
    const size_t qb = (size_t)h->c.q_order * h->n * (h->c.q_bf16 ? 2 : 4);
    CK(cudaMemsetAsync(h->wq[0], 0, qb, h->st));
    CK(cudaMemsetAsync(h->wq[1], 0, qb, h->st));
  }
  if (h->ext.out) CK(cudaMemsetAsync(h->ext.out, 0, (size_t)h->ext.ntr * h->ext.nt * 4, h->st));
  h->iq0 = 0;
  return RTM_OK;
}

static QDev q_dev(Engine *h) {
  QDev q{};
  q.order = h->c.q_order;
  q.cqsum = h->cqsum;
  for (int l = 0; l < q.order && l < 8; l++) q.cq[l] = h->cq[l], q.wq[l] = h->cwq[l];
  q.invq = h->invq;
  q.d0 = h->wq[h->iq0];
  q.d1 = h->wq[1 - h->iq0];
  q.bf16 = h->c.q_bf16 ? 1 : 0;
  return q;
}

// One application of the spatial operator, optionally fused with update2nd
// (mode 1 leapfrog, 2 Q) and with the snapshot / imaging access of the
// previous step's wavefield (io).
// Engine CFD on a 3-D grid: the segment-parallel fused pipeline (five
// launches: Z(w1), X(w1), the fused y kernel, Z(pz), the fused x kernel).
static int cfd_seg_step(Engine *h, int mode, const QDev &q) {
  const rtm_dims &d = h->d;
  CfdSegArgs a{};
  a.nx = d.nx, a.ny = d.ny, a.nz = d.nz, a.pml3d = h->c.pml3d, a.model = h->c.model_type, a.mode = mode;
  a.pml = pml_dev(h);
  a.q = q;
  a.w1 = h->w1, a.w0 = h->w0, a.vel = h->vel;
  a.eps = h->eps, a.del = h->del, a.pjx = h->pjx, a.pjy = h->pjy, a.rho = h->rho;
  a.gx = h->px, a.gz = h->pz, a.dz = h->scr2, a.dy = h->scr;
  CUtensorMap mx1, my1, mxp;
  bool tx1 = false, ty1 = false, txp = false;
  if (h->cfd_xy == 3 && h->cfd_tma) {
    int Rx, nbx, Ry, nby;
    cfd_tma_box(d.nx, &Rx, &nbx);
    cfd_tma_box(d.ny, &Ry, &nby);
    tx1 = tmap(h, h->w1, 32, Rx, &mx1);
    ty1 = tmap(h, h->w1, 32, 1, &my1, Ry);
    txp = tmap(h, h->px, 32, Rx, &mxp);
  }
  {
    KScope k(h, RTM_K_CFD_Z);
    launch_cfd_seg_line(DZ, 0, h->cfd[DZ][0], h->w1, h->pz, a, nullptr, h->dflag, h->st);
  }
  {
    KScope k(h, RTM_K_CFD_X);
    launch_cfd_seg_line(DX, 0, h->cfd[DX][0], h->w1, h->px, a, tx1 ? &mx1 : nullptr, h->dflag, h->st);
  }
  {
    KScope k(h, RTM_K_CFD_YF);
    launch_cfd_seg_yfused(h->cfd[DY][0], h->cfd[DY][1], a, ty1 ? &my1 : nullptr, h->dflag, h->st);
  }
  {
    KScope k(h, RTM_K_CFD_Z);
    launch_cfd_seg_line(DZ, 1, h->cfd[DZ][1], h->pz, h->scr2, a, nullptr, h->dflag, h->st);
  }
  {
    KScope k(h, RTM_K_CFD_XF);
    launch_cfd_seg_xfused(h->cfd[DX][1], a, txp ? &mxp : nullptr, h->dflag, h->st);
  }
  return check_launch(h, "cfd_seg_step");
}

static int step_kernel(Engine *h, int mode, const FusedIo &io) {
  const rtm_dims &d = h->d;
  QDev q = q_dev(h);
  if (h->lap_iso()) {
    IsoArgs a{};
    a.nx = d.nx, a.ny = d.ny, a.nz = d.nz, a.yseg = h->yseg;
    a.w1 = h->w1, a.w0 = h->w0, a.vel = h->vel;
    memcpy(a.c2x, h->c2x, sizeof a.c2x), memcpy(a.c2y, h->c2y, sizeof a.c2y), memcpy(a.c2z, h->c2z, sizeof a.c2z);
    a.pml = pml_dev(h);
    a.io = io;
    a.q = q;
    CUtensorMap m1, m0, mv;
    if (h->iso4 == 2) {
      const int tx = kIso4TmaShapes[h->v4_shape].tx;
      if (!h->t_iso.current(tx, h->v4_yseg)) {
        h->err = "iso4 tile table is stale";
        return RTM_ERR_STATE;
      }
      if (!tmap(h, h->w1, 40, tx + 8, &m1) || !tmap(h, h->w0, 32, tx, &m0) || !tmap(h, h->vel, 32, tx, &mv)) {
        h->iso4 = 1;
        h->v4_yseg = yseg_iso4(h);
      }
    }
    if (h->iso4) {
      a.yseg = h->v4_yseg;
      if (h->iso4 == 2) {
        {
          const TileSet &t = h->t_iso;
          KScope k(h, RTM_K_ISO, (t.n_int > 0) + (t.n_edge > 0));
          launch_iso_fd8_tma4(a, t.d, t.n_int, false, m1, m0, mv, h->dflag, mode, h->c.pml3d, h->v4_shape, h->st);
          launch_iso_fd8_tma4(a, t.d + t.n_int, t.n_edge, true, m1, m0, mv, h->dflag, mode, h->c.pml3d, h->v4_shape,
                              h->st);
        }
        return check_launch(h, "iso_fd8_tma4");
      }
      {
        KScope k(h, RTM_K_ISO);
        launch_iso_fd8_v4(a, mode, h->c.pml3d, h->v4_tx, h->st);
      }
      return check_launch(h, "iso_fd8_v4");
    }
    if (h->use_tma) {
      const int tx = kIsoTmaShapes[h->tma_shape].tx;
      if (!tmap(h, h->w1, 40, tx + 8, &m1) || !tmap(h, h->w0, 32, tx, &m0) || !tmap(h, h->vel, 32, tx, &mv))
        h->use_tma = 0;
      else a.yseg = yseg_for(h, tx);
    }
    {
      KScope k(h, RTM_K_ISO);
      if (h->use_tma) launch_iso_fd8_tma(a, m1, m0, mv, h->dflag, mode, h->c.pml3d, h->tma_shape, h->st);
      else launch_iso_fd8(a, mode, h->c.pml3d, h->tx, h->st);
    }
    return check_launch(h, "iso_fd8_step");
  }
  if (h->c.engine == RTM_ENGINE_FD8 && h->aniso4) {
    const TileSet &t = h->t_an4;
    if (!t.current(kAniso4TX, h->an4_yseg)) {
      h->err = "FD8 4-cell tile table is stale";
      return RTM_ERR_STATE;
    }
    GradArgs g{};
    g.nx = d.nx, g.ny = d.ny, g.nz = d.nz, g.yseg = h->an4_yseg, g.pml3d = h->c.pml3d;
    g.w1 = h->w1, g.px = h->px, g.py = h->py, g.pz = h->pz;
    g.eps = h->eps, g.del = h->del, g.pjx = h->pjx, g.pjy = h->pjy;
    memcpy(g.c1x, h->c1x, sizeof g.c1x), memcpy(g.c1y, h->c1y, sizeof g.c1y), memcpy(g.c1z, h->c1z, sizeof g.c1z);
    g.pml = pml_dev(h);
    g.io = io;
    DivArgs v{};
    v.nx = d.nx, v.ny = d.ny, v.nz = d.nz, v.yseg = h->an4_yseg, v.pml3d = h->c.pml3d;
    v.px = h->px, v.py = h->py, v.pz = h->pz, v.w1 = h->w1, v.w0 = h->w0, v.vel = h->vel;
    memcpy(v.c1x, h->c1x, sizeof v.c1x), memcpy(v.c1y, h->c1y, sizeof v.c1y), memcpy(v.c1z, h->c1z, sizeof v.c1z);
    v.pml = pml_dev(h);
    v.q = q;
    const int T = kAniso4TX;
    Grad4Maps gm;
    Div4Maps dm;
    const bool tti = h->c.model_type == RTM_TTI;
    bool ok = tmap(h, h->w1, 40, T + 8, &gm.w1) && tmap(h, h->eps, 32, T, &gm.m[0]) && tmap(h, h->del, 32, T, &gm.m[1]);
    gm.m[2] = gm.m[3] = gm.m[0];
    if (tti) ok = ok && tmap(h, h->pjx, 32, T, &gm.m[2]) && (!h->pjy || tmap(h, h->pjy, 32, T, &gm.m[3]));
    ok = ok && tmap(h, h->px, 32, T + 8, &dm.px) && tmap(h, h->pz, 40, T, &dm.pz) &&
         tmap(h, h->py ? h->py : h->px, 32, T, &dm.py) && tmap(h, h->w0, 32, T, &dm.w0) &&
         tmap(h, h->vel, 32, T, &dm.vel) && tmap(h, h->w1, 32, T, &dm.w1);
    // the visco-acoustic update takes its Q memory and 1/Q from ring B when
    // they fit it (order <= kDiv4QMax; BF16 rows need nz % 8 == 0)
    dm.qring = 0;
    if (ok && mode == 2 && h->c.q_order <= kDiv4QMax && h->qring_ok &&
        tmap_q(h, q.d0, T, &dm.qa) && tmap_q(h, q.d1, T, &dm.qb) && tmap(h, h->invq, 32, T, &dm.iq))
      dm.qring = h->c.q_bf16 ? 2 : 1;
    if (ok) {
      {
        KScope k(h, RTM_K_GRAD, (t.n_int > 0) + (t.n_edge > 0));
        launch_grad4(g, t.d, t.n_int, false, h->c.model_type, gm, h->dflag, h->st);
        launch_grad4(g, t.d + t.n_int, t.n_edge, true, h->c.model_type, gm, h->dflag, h->st);
      }
      TRY(check_launch(h, "grad4"));
      {
        KScope k(h, RTM_K_DIV, (t.n_int > 0) + (t.n_edge > 0));
        launch_div4(v, t.d, t.n_int, false, mode, dm, h->dflag, h->st);
        launch_div4(v, t.d + t.n_int, t.n_edge, true, mode, dm, h->dflag, h->st);
      }
      return check_launch(h, "div4");
    }
    h->aniso4 = 0;  // tensor maps unavailable: the one-cell passes below
  }
  if (h->c.engine == RTM_ENGINE_FD8) {
    const TileSet &t = h->t_fd8;
    if (!t.current(h->tx, h->yseg)) {
      h->err = "FD8 tile table is stale";
      return RTM_ERR_STATE;
    }
    GradArgs g{};
    g.nx = d.nx, g.ny = d.ny, g.nz = d.nz, g.yseg = h->yseg, g.pml3d = h->c.pml3d;
    g.w1 = h->w1, g.px = h->px, g.py = h->py, g.pz = h->pz;
    g.h = StateF16{h->h1, h->s1, h->h0, h->s0, h->sn, h->m0};
    g.eps = h->eps, g.del = h->del, g.pjx = h->pjx, g.pjy = h->pjy, g.rho = h->rho;
    memcpy(g.c1x, h->c1x, sizeof g.c1x), memcpy(g.c1y, h->c1y, sizeof g.c1y), memcpy(g.c1z, h->c1z, sizeof g.c1z);
    g.pml = pml_dev(h);
    g.io = io;
    {
      KScope k(h, RTM_K_GRAD, (t.n_int > 0) + (t.n_edge > 0));
      launch_grad_fd8(g, t.d, t.n_int, false, h->c.model_type, h->tx, h->st, h->f16);
      launch_grad_fd8(g, t.d + t.n_int, t.n_edge, true, h->c.model_type, h->tx, h->st, h->f16);
    }
    TRY(check_launch(h, "grad_fd8"));
    if (h->f16) {  // scale of the field this step writes, then its fresh slab maxima
      launch_f16_scales(h->m0, h->m1, h->sn, d.ny, h->f16_floor, h->st);
      CK(cudaMemsetAsync(h->m0, 0, d.ny * 4, h->st));
    }
    DivArgs v{};
    v.nx = d.nx, v.ny = d.ny, v.nz = d.nz, v.yseg = h->yseg, v.pml3d = h->c.pml3d;
    v.h = StateF16{h->h1, h->s1, h->h0, h->s0, h->sn, h->m0};
    v.px = h->px, v.py = h->py, v.pz = h->pz, v.w1 = h->w1, v.w0 = h->w0, v.vel = h->vel, v.rho = h->rho;
    memcpy(v.c1x, h->c1x, sizeof v.c1x), memcpy(v.c1y, h->c1y, sizeof v.c1y), memcpy(v.c1z, h->c1z, sizeof v.c1z);
    v.pml = pml_dev(h);
    v.q = q;
    {
      KScope k(h, RTM_K_DIV, (t.n_int > 0) + (t.n_edge > 0));
      launch_div_fd8(v, t.d, t.n_int, false, mode, h->tx, h->st, h->f16);
      launch_div_fd8(v, t.d + t.n_int, t.n_edge, true, mode, h->tx, h->st, h->f16);
    }
    return check_launch(h, "div_fd8");
  }
  // compact FD: raw line-solve derivatives, then pointwise PML / scaling /
  // accumulation epilogues (FdEngine_cfd + KernelCPU::TTI structure)
  if (io.store || io.ic) {
    KScope k(h, RTM_K_IO);
    launch_fused_io(io, h->w1, d.nx, d.ny, d.nz, h->st);
  }
  TRY(check_launch(h, "fused_io"));
  if (h->cfd_xy == 3 || h->cfd_xy == 4) return cfd_seg_step(h, mode, q);
  // the z line solve fused with the epilogue's interior box (x / y first):
  // compact-FD line solves only (not the transform engines), not the
  // visco-acoustic update of the divergence pass
  const bool zfuse = h->cfd_zfuse && !h->fft && !h->r2r;
  if (!zfuse) {
    KScope k(h, RTM_K_CFD_Z);
    cfd_deriv(h, DZ, 0, h->w1, h->pz);
  }
  {
    KScope k(h, RTM_K_CFD_X);
    cfd_deriv(h, DX, 0, h->w1, h->px);
  }
  if (d.ny > 1) {
    KScope k(h, RTM_K_CFD_Y);
    cfd_deriv(h, DY, 0, h->w1, h->py);
  }
  TRY(check_launch(h, "cfd_deriv(grad)"));
  CfdGradEpiArgs ge{};
  ge.nx = d.nx, ge.ny = d.ny, ge.nz = d.nz, ge.pml3d = h->c.pml3d, ge.model = h->c.model_type;
  ge.gx = h->px, ge.gy = h->py, ge.gz = h->pz;
  ge.eps = h->eps, ge.del = h->del, ge.pjx = h->pjx, ge.pjy = h->pjy, ge.rho = h->rho;
  ge.pml = pml_dev(h);
  {
    KScope k(h, RTM_K_CFD_GEPI);
    if (zfuse) launch_cfd_zgrad(h->cfd[DZ][0], h->w1, ge, h->st);
    else launch_cfd_grad_epilogue(ge, h->st);
  }
  TRY(check_launch(h, "cfd_grad_epilogue"));
  // divergence parts: d/dx px -> scr2, d/dz pz -> scr, d/dy py -> px (px is free now)
  const bool zfuse_div = zfuse && mode != 2;
  {
    KScope k(h, RTM_K_CFD_X);
    cfd_deriv(h, DX, 1, h->px, h->scr2);
  }
  float *dzp = h->scr;
  if (!zfuse_div) {
    KScope k(h, RTM_K_CFD_Z);
    cfd_deriv(h, DZ, 1, h->pz, dzp);
  }
  float *dyp = nullptr;
  if (d.ny > 1) {
    KScope k(h, RTM_K_CFD_Y);
    cfd_deriv(h, DY, 1, h->py, h->px);
    dyp = h->px;
  }
  TRY(check_launch(h, "cfd_deriv(div)"));
  CfdDivEpiArgs de{};
  de.nx = d.nx, de.ny = d.ny, de.nz = d.nz, de.pml3d = h->c.pml3d, de.mode = mode;
  de.dx = h->scr2, de.dz = dzp, de.dy = dyp;
  de.w1 = h->w1, de.w0 = h->w0, de.vel = h->vel, de.rho = h->rho;
  de.rho_form = (h->c.engine == RTM_ENGINE_CFDB || h->c.engine == RTM_ENGINE_FFTV || h->c.engine == RTM_ENGINE_SINCOS)
                    ? 2
                : (h->c.engine == RTM_ENGINE_R2C || h->c.engine == RTM_ENGINE_R2R) ? 1
                                                                                    : 0;
  de.pml = pml_dev(h);
  de.q = q;
  {
    KScope k(h, RTM_K_CFD_DEPI);
    if (zfuse_div) {
      // the Derivative path's divergence pass takes plan iswitch (cfd_deriv)
      const bool deriv_path = h->c.engine == RTM_ENGINE_CFDB;
      launch_cfd_zdiv(h->cfd[DZ][deriv_path && h->c.model_type == RTM_TTI ? 0 : 1], h->pz, de, h->st);
    } else {
      launch_cfd_div_epilogue(de, h->st);
    }
  }
  return check_launch(h, "cfd_div_epilogue");
}

static int do_inject(Engine *h, int it) {
  TraceSetDev &t = h->inj;
  if (!t.ntr || it < 0 || it >= t.nt) return RTM_OK;
  TraceDev td = t.dev();
  if (h->f16) {
    KScope k(h, RTM_K_INJECT);
    launch_inject_scatter_f16(td, it, h->h0, h->sn, h->m0, h->vel, h->d.nx, h->d.ny, h->d.nz, h->st);
    return check_launch(h, "inject");
  }
  KScope k(h, RTM_K_INJECT, (int)t.groups.size() + (t.n_ungrouped ? 1 : 0));
  for (const GroupDev &g : t.groups)
    launch_inject_group(g, td, it, h->plane, h->w0, h->vel, h->d.nx, h->d.ny, h->d.nz, h->st);
  if (t.n_ungrouped) {
    td.ids = t.ungrouped, td.nids = t.n_ungrouped;
    launch_inject_scatter(td, it, h->w0, h->vel, h->d.nx, h->d.ny, h->d.nz, h->st);
  }
  return check_launch(h, "inject");
}

static int do_extract(Engine *h, int jt) {
  TraceSetDev &t = h->ext;
  if (!t.ntr || jt < 0 || jt >= t.nt) return RTM_OK;
  TraceDev td = t.dev();
  if (h->f16) {
    KScope k(h, RTM_K_EXTRACT);
    launch_extract_direct_f16(td, h->h0, h->sn, t.out, jt, t.nt, h->d.nx, h->d.ny, h->d.nz, h->st);
    return check_launch(h, "extract");
  }
  KScope k(h, RTM_K_EXTRACT, 2 * (int)t.groups.size() + (t.n_ungrouped ? 1 : 0));
  for (const GroupDev &g : t.groups)
    launch_extract_group(g, td, h->w0, h->plane, t.out, jt, t.nt, h->d.nx, h->d.ny, h->d.nz, h->st);
  if (t.n_ungrouped) {
    td.ids = t.ungrouped, td.nids = t.n_ungrouped;
    launch_extract_direct(td, h->w0, t.out, jt, t.nt, h->d.nx, h->d.ny, h->d.nz, h->st);
  }
  return check_launch(h, "extract");
}

static void do_swap(Engine *h) {
  std::swap(h->w0, h->w1);
  h->iq0 = 1 - h->iq0;
  if (h->f16) {  // the new field (scale sn) becomes w1, the old w1 (scale s1) becomes w0
    std::swap(h->h0, h->h1);
    float *t = h->s0;
    h->s0 = h->s1, h->s1 = h->sn, h->sn = t;
    std::swap(h->m0, h->m1);
  }
}

// FP32 copy of an FP16 state field in the px scratch: which = 0 / 1 the w0 /
// w1 of a completed step, 2 the field the current step wrote (before the swap)
static float *f16_view(Engine *h, int which) {
  const __half *f = which == 1 ? h->h1 : h->h0;
  const float *sc = which == 0 ? h->s0 : which == 1 ? h->s1 : h->sn;
  launch_f16_to_f32(f, sc, h->px, h->d.ny, h->nxz, h->st);
  return h->px;
}

static SnapDev slot_dev(Engine *h, int slot) {
  SnapDev s{};
  s.fmt = h->snap_fmt;
  s.base = h->snaps + (size_t)(h->nstage ? slot % h->nstage : slot) * h->slot_bytes;
  s.slab = h->slabs ? h->slabs + (size_t)slot * h->d.ny : nullptr;
  return s;
}

static FusedIo io_none() { return FusedIo{}; }

static FusedIo io_store(Engine *h, int slot) {
  FusedIo io{};
  io.store = 1;
  io.st = slot_dev(h, slot);
  return io;
}

static FusedIo io_image(Engine *h, int slot) {
  FusedIo io{};
  io.ic = 1;
  io.src = slot_dev(h, slot);
  io.image = h->image, io.comp = h->comp;
  // the time taper follows the snapshot's place in the shot, not its slot
  const int snap = slot + h->slot0;
  io.use_t = snap >= 0 && snap < (int)h->taper_t.size();
  io.tscale = io.use_t ? h->taper_t[snap] : 1.f;
  io.taper_z = h->taper_z;
  io.ex = h->ic_edge ? h->ex : h->one_x;
  io.ey = h->ic_edge ? h->ey : h->one_y;
  io.ez = h->ic_edge ? h->ez : h->one_z;
  io.illum = h->illum_on ? h->illum : nullptr;
  return io;
}

// learned-compressor slot: latents [nb][64] (bfloat16, 128 bytes per block), then scales [nb]
static float *ae_latent(Engine *h, int slot) { return (float *)(h->snaps + (size_t)slot * h->slot_bytes); }
static float *ae_scales(Engine *h, int slot) {
  return ae_latent(h, slot) + (size_t)ae_volume_blocks(h->d.nx, h->d.ny, h->d.nz) * 32;
}
// fallback blocks per slot and the slot's fallback area (after latents and scales)
static long long ae_fb_cap(Engine *h) {
  const long long nb = ae_volume_blocks(h->d.nx, h->d.ny, h->d.nz);
  return h->ae_fb_frac > 0.f ? std::max(1LL, (long long)std::ceil((double)h->ae_fb_frac * nb)) : 0;
}
static void *ae_fb(Engine *h, int slot) {
  const size_t lat = ((size_t)ae_volume_blocks(h->d.nx, h->d.ny, h->d.nz) * 33 * 4 + 15) / 16 * 16;
  return (char *)ae_latent(h, slot) + lat;
}
static int ae_store(Engine *h, int slot, const float *w) {
  KScope k(h, RTM_K_IO);
  TRY(ae_compress(h->ae, w, h->d.nx, h->d.ny, h->d.nz, ae_latent(h, slot), ae_scales(h, slot), h->st));
  if (const long long cap = ae_fb_cap(h))
    ae_fallback_store(w, ae_scales(h, slot), h->d.nx, h->d.ny, h->d.nz, h->ae_fb_tau, cap, ae_fb(h, slot), h->st);
  return check_launch(h, "ae_compress");
}
static int ae_load(Engine *h, int slot, float *w) {
  KScope k(h, RTM_K_IO);
  TRY(ae_decompress(h->ae, ae_latent(h, slot), ae_scales(h, slot), h->d.nx, h->d.ny, h->d.nz, w, h->st));
  if (const long long cap = ae_fb_cap(h))
    ae_fallback_apply(ae_scales(h, slot), h->d.nx, h->d.ny, h->d.nz, cap, ae_fb(h, slot), w, h->st);
  return check_launch(h, "ae_decompress");
}
// imaging-condition term with the source snapshot decoded into ae_scratch
static FusedIo io_image_ae(Engine *h, int slot) {
  FusedIo io = io_image(h, slot);
  io.src = SnapDev{RTM_SNAP_FP32, h->ae_scratch, nullptr};
  return io;
}

// INVERSION imaging term of slot `slot` against receiver field u, at once
static int ic_explicit(Engine *h, int slot, const float *u) {
  const FusedIo io = h->snap_fmt == RTM_SNAP_AE ? io_image_ae(h, slot) : io_image(h, slot);
  KScope k(h, RTM_K_IO, 10);
  if (launch_ic_inversion(h->ic_plans, io, u, h->icS, h->icR, h->icDs, h->icDr, h->icSh, h->icRh, h->icTh, h->d.nx,
                          h->d.ny, h->d.nz, h->d.dx, h->d.dy, h->d.dz, h->st)) {
    h->err = "cuFFT execution failed";
    return RTM_ERR_CUDA;
  }
  return check_launch(h, "ic_inversion");
}

// double-grid IMAGE1 term of slot `slot` against receiver field u, at once
static int ic_double_explicit(Engine *h, int slot, const float *u) {
  const FusedIo io = h->snap_fmt == RTM_SNAP_AE ? io_image_ae(h, slot) : io_image(h, slot);
  KScope k(h, RTM_K_IO, 12);
  const int rc = launch_ic_double(h->dbl_fft, h->dmap, io, u, h->dblS, h->dblR, h->dbl_img, h->dbl_comp,
                                  h->illum_on ? h->illum : nullptr, h->d.nx, h->d.ny, h->d.nz, h->dbl_hz, h->dbl_hxy,
                                  h->st);
  if (rc != RTM_OK) {
    h->err = "double-grid imaging: a line transform failed";
    return rc;
  }
  return check_launch(h, "ic_double");
}

// per-slot slab statistics for the 16-bit formats, taken on w0 after injection
static int snap_prepare(Engine *h, int slot) {
  if (h->snap_fmt == RTM_SNAP_FP32 || h->snap_fmt == RTM_SNAP_AE) return RTM_OK;
  SnapDev s = slot_dev(h, slot);
  KScope k(h, RTM_K_SLAB);
  if (h->f16) {
    launch_f16_slab_hdr(h->m0, (float *)s.slab, h->snap_fmt == RTM_SNAP_C16 ? (uint16_t *)s.base : nullptr,
                        h->snap_fmt, h->d.nx, h->d.ny, h->d.nz, h->st);
    return check_launch(h, "slab_hdr");
  }
  launch_slab_max(h->w0, (float *)s.slab, h->snap_fmt == RTM_SNAP_C16 ? (uint16_t *)s.base : nullptr, h->snap_fmt,
                  h->d.nx, h->d.ny, h->d.nz, h->st);
  return check_launch(h, "slab_max");
}

// ---- snapshot offload: copies between host slots and device staging slots ----
// (all on st_copy; st forks to it with ev_fork and waits for stage_ev[k])
static int stage_fork(Engine *h) {
  CK(cudaEventRecord(h->ev_fork, h->st));
  CK(cudaStreamWaitEvent(h->st_copy, h->ev_fork, 0));
  return RTM_OK;
}
// slot s (just written to its staging slot by work already on st) to the host
static int offload_d2h(Engine *h, int s) {
  const int k = s % h->nstage;
  TRY(stage_fork(h));
  CK(cudaMemcpyAsync(h->host_snaps + (size_t)s * h->slot_bytes, h->snaps + (size_t)k * h->slot_bytes, h->slot_bytes,
                     cudaMemcpyDeviceToHost, h->st_copy));
  CK(cudaEventRecord(h->stage_ev[k], h->st_copy));
  h->stage_slot[k] = -1, h->stage_wait[k] = true;
  return RTM_OK;
}
// slot s from the host into its staging slot (after every kernel already on st)
static int offload_h2d(Engine *h, int s) {
  const int k = s % h->nstage;
  TRY(stage_fork(h));
  CK(cudaMemcpyAsync(h->snaps + (size_t)k * h->slot_bytes, h->host_snaps + (size_t)s * h->slot_bytes, h->slot_bytes,
                     cudaMemcpyHostToDevice, h->st_copy));
  CK(cudaEventRecord(h->stage_ev[k], h->st_copy));
  h->stage_slot[k] = s, h->stage_wait[k] = true;
  return RTM_OK;
}
// st waits for the last copy into / out of the staging slot of s
static int stage_ready(Engine *h, int s) {
  const int k = s % h->nstage;
  if (h->stage_wait[k]) CK(cudaStreamWaitEvent(h->st, h->stage_ev[k], 0));
  h->stage_wait[k] = false;
  return RTM_OK;
}
// join every copy back into st (before a graph capture ends, and after a loop)
static int stage_join(Engine *h) {
  if (!h->nstage) return RTM_OK;
  for (int k = 0; k < h->nstage; k++) TRY(stage_ready(h, k));
  return RTM_OK;
}

// Runs fn(step index) for `count` steps inside CUDA graphs of up to `chunk`
// steps each, timed with events on the engine's stream; every snapshot copy
// forked from the engine stream is joined back before a capture ends.
template <typename F> static int run_graphs(Engine *h, int count, F fn) {
  const int chunk = 256;
  h->launches = 0;
  CK(cudaEventRecord(h->ev0, h->st));
  if (h->prof_on) {  // eager launches bracketed by events (no graph)
    for (int s = 0; s < count; s++) TRY(fn(s));
    TRY(stage_join(h));
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaEventSynchronize(h->ev1));
    CK(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
    prof_collect(h);
    return check_flag(h);
  }
  for (int s0 = 0; s0 < count; s0 += chunk) {
    const int s1 = std::min(count, s0 + chunk);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int rc = RTM_OK;
    for (int s = s0; s < s1 && rc == RTM_OK; s++) rc = fn(s);
    if (rc == RTM_OK) rc = stage_join(h);
    cudaError_t ec = cudaStreamEndCapture(h->st, &g);
    if (rc != RTM_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture", h);
    cudaGraphExec_t ge = nullptr;
    cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate", h);
    cudaError_t el = cudaGraphLaunch(ge, h->st);
    cudaGraphExecDestroy(ge);
    if (el != cudaSuccess) return cuda_fail(el, "cudaGraphLaunch", h);
  }
  CK(cudaEventRecord(h->ev1, h->st));
  CK(cudaEventSynchronize(h->ev1));
  CK(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  return check_flag(h);
}

static int ready(Engine *h) {
  if (!h) return RTM_ERR_ARG;
  if (!h->model_set) {
    h->err = "rtm_set_model has not been called";
    return RTM_ERR_STATE;
  }
  cudaSetDevice(h->device);
  return RTM_OK;
}

// Host staging of the traces of a TraceSet and its grouping by z kernel.
static int upload_traces(Engine *h, TraceSetDev &t, int ntr, int lx, int ly, int lz, const int *off3, const int *len3,
                         const float *kx, const float *ky, const float *kz, const float *traces, int nt, float scaler,
                         bool extraction) {
  for (void *p : {(void *)t.off, (void *)t.len, (void *)t.kx, (void *)t.ky, (void *)t.kz, (void *)t.traces,
                  (void *)t.out, (void *)t.ungrouped})
    h->release(p);
  for (void *p : t.group_allocs) h->release(p);
  t = TraceSetDev{};
  if (ntr <= 0) return RTM_OK;
  // validate every kernel box against the grid
  for (int r = 0; r < ntr; r++) {
    const int *o = off3 + 3 * r, *l = len3 + 3 * r;
    const int nn[3] = {h->d.nx, h->d.ny, h->d.nz}, cap[3] = {lx, ly, lz};
    for (int a = 0; a < 3; a++)
      if (l[a] < 0 || l[a] > cap[a] || o[a] < 0 || o[a] + l[a] > nn[a]) {
        h->err = "trace " + std::to_string(r) + " kernel box outside the grid or its stride";
        return RTM_ERR_ARG;
      }
  }
  t.ntr = ntr, t.lx = lx, t.ly = ly, t.lz = lz, t.nt = nt, t.scaler = scaler;
  TRY(h->alloc(t.off, 3 * (size_t)ntr));
  TRY(h->alloc(t.len, 3 * (size_t)ntr));
  TRY(h->alloc(t.kx, (size_t)ntr * lx));
  TRY(h->alloc(t.ky, (size_t)ntr * ly));
  TRY(h->alloc(t.kz, (size_t)ntr * lz));
  CK(cudaMemcpy(t.off, off3, 12 * (size_t)ntr, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(t.len, len3, 12 * (size_t)ntr, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(t.kx, kx, 4 * (size_t)ntr * lx, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(t.ky, ky, 4 * (size_t)ntr * ly, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(t.kz, kz, 4 * (size_t)ntr * lz, cudaMemcpyHostToDevice));
  if (!extraction) {
    TRY(h->alloc(t.traces, (size_t)ntr * nt));
    CK(cudaMemcpy(t.traces, traces, 4 * (size_t)ntr * nt, cudaMemcpyHostToDevice));
  } else {
    TRY(h->alloc(t.out, (size_t)ntr * nt));
    CK(cudaMemset(t.out, 0, 4 * (size_t)ntr * nt));
  }
  // group traces whose z kernels are identical (first index, length, values)
  std::map<std::vector<uint32_t>, std::vector<int>> by_z;
  for (int r = 0; r < ntr; r++) {
    std::vector<uint32_t> key;
    key.push_back((uint32_t)off3[3 * r + 2]);
    key.push_back((uint32_t)len3[3 * r + 2]);
    for (int k = 0; k < len3[3 * r + 2]; k++) {
      uint32_t b;
      memcpy(&b, kz + (size_t)r * lz + k, 4);
      key.push_back(b);
    }
    by_z[key].push_back(r);
  }
  std::vector<int> loose;
  const int T = 16;
  for (auto &kv : by_z) {
    const std::vector<int> &mem = kv.second;
    if (mem.size() < 16) {
      loose.insert(loose.end(), mem.begin(), mem.end());
      continue;
    }
    const int r0 = mem[0];
    GroupDev g{};
    g.ntr = (int)mem.size();
    g.offz = off3[3 * r0 + 2];
    g.lz = len3[3 * r0 + 2];
    g.tile = T;
    const int ntx = (h->d.nx + T - 1) / T, nty = (h->d.ny + T - 1) / T;
    std::vector<std::vector<int>> lists((size_t)ntx * nty);
    for (int r : mem) {
      const int *o = off3 + 3 * r, *l = len3 + 3 * r;
      if (!l[0] || !l[1]) continue;
      for (int ty = o[1] / T; ty <= (o[1] + l[1] - 1) / T; ty++)
        for (int tx = o[0] / T; tx <= (o[0] + l[0] - 1) / T; tx++) lists[(size_t)ty * ntx + tx].push_back(r);
    }
    std::vector<int> txy, ptr{0}, lst;
    for (int ty = 0; ty < nty; ty++)
      for (int tx = 0; tx < ntx; tx++) {
        auto &L = lists[(size_t)ty * ntx + tx];
        if (L.empty()) continue;
        txy.push_back(tx * T), txy.push_back(ty * T);
        lst.insert(lst.end(), L.begin(), L.end());
        ptr.push_back((int)lst.size());
      }
    g.ntiles = (int)txy.size() / 2;
    int *dm, *dxy, *dp, *dl;
    float *dkz;
    TRY(h->alloc(dm, mem.size()));
    TRY(h->alloc(dkz, std::max(1, g.lz)));
    TRY(h->alloc(dxy, std::max<size_t>(2, txy.size())));
    TRY(h->alloc(dp, ptr.size()));
    TRY(h->alloc(dl, std::max<size_t>(1, lst.size())));
    t.group_allocs.insert(t.group_allocs.end(), {dm, dkz, dxy, dp, dl});
    CK(cudaMemcpy(dm, mem.data(), 4 * mem.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dkz, kz + (size_t)r0 * lz, 4 * g.lz, cudaMemcpyHostToDevice));
    if (!txy.empty()) CK(cudaMemcpy(dxy, txy.data(), 4 * txy.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dp, ptr.data(), 4 * ptr.size(), cudaMemcpyHostToDevice));
    if (!lst.empty()) CK(cudaMemcpy(dl, lst.data(), 4 * lst.size(), cudaMemcpyHostToDevice));
    g.members = dm, g.kz = dkz, g.tile_xy = dxy, g.tile_ptr = dp, g.tile_list = dl;
    t.groups.push_back(g);
  }
  if (!loose.empty()) {
    TRY(h->alloc(t.ungrouped, loose.size()));
    CK(cudaMemcpy(t.ungrouped, loose.data(), 4 * loose.size(), cudaMemcpyHostToDevice));
    t.n_ungrouped = (int)loose.size();
  }
  if (!t.groups.empty() && !h->plane) TRY(h->alloc(h->plane, (size_t)h->d.nx * h->d.ny));
  return RTM_OK;
}

static void edge_taper(int n, int nt, std::vector<float> &w) {
  // decode tapers of bgprtm/WaveFieldCompress.cpp:88-98 and 189-200
  w.assign(n, 1.0f);
  if (n <= 2 * nt) return;
  for (int i = 0; i < nt; i++) {
    float v = 0.5f * (1.0f - cosf((float)M_PI * float(i) / float(nt)));
    w[i] = v;
    w[n - 1 - i] = v;
  }
}

}  // namespace rtm

using rtm::Engine;

struct rtm_handle : Engine {};

// ---- batched small shots ----------------------------------------------------
struct rtm_batch {
  std::vector<rtm::Engine *> shots;
  int device = 0, pml3d = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  int tx = 8, yseg = 0;  // tile width, y segment (0: whole y extent)
  rtm::IsoBatchShot *d_shots = nullptr;    // every shot's I/O (and ISO step) arguments
  rtm::AnisoBatchShot *d_ashots = nullptr;  // VTI / TTI batches: the two passes' arguments
  int *d_start = nullptr;
  int cap = 0;
  int model = RTM_ISO;  // the shots' model type (ISO: one-pass kernel; VTI / TTI: two passes)
  std::string err;
};

namespace rtm {
// tile-shape candidates of the batched kernels: {tile width, y segment (0 =
// whole y)}; the VTI / TTI passes take those of width kAnisoBatchTX
static const int kBatchShapes[][2] = {{8, 0}, {8, 32}, {16, 0}, {16, 32}, {8, 16}};
static const int kBatchNShapes = 5;

// Device table of the shots in `order`, their first work items, and the
// trace maxima of the batched I/O launches.
static int batch_upload(rtm_batch *b, const std::vector<int> &order, std::vector<int> &start, int &max_inj,
                        int &max_ly, int &max_ext) {
  const int n = (int)order.size();
  const bool aniso = b->model != RTM_ISO;
  const int tx = aniso ? kAnisoBatchTX : b->tx;
  std::vector<IsoBatchShot> hs(n);
  std::vector<AnisoBatchShot> ha(aniso ? n : 0);
  start.assign(n + 1, 0);
  max_inj = max_ly = max_ext = 0;
  for (int k = 0; k < n; k++) {
    Engine *h = b->shots[order[k]];
    const rtm_dims &d = h->d;
    IsoBatchShot &S = hs[k];
    IsoArgs &a = S.a;
    a.nx = d.nx, a.ny = d.ny, a.nz = d.nz;
    a.yseg = b->yseg > 0 ? std::min(b->yseg, d.ny) : d.ny;
    a.w1 = h->w1, a.w0 = h->w0, a.vel = h->vel;
    memcpy(a.c2x, h->c2x, sizeof a.c2x), memcpy(a.c2y, h->c2y, sizeof a.c2y), memcpy(a.c2z, h->c2z, sizeof a.c2z);
    a.pml = pml_dev(h);
    a.io = FusedIo{};
    a.q = QDev{};
    S.wa = h->w1, S.wb = h->w0;
    S.tiles_z = (d.nz + 31) / 32, S.tiles_x = (d.nx + tx - 1) / tx, S.tiles_y = (d.ny + a.yseg - 1) / a.yseg;
    S.inj = h->inj.dev(), S.ext = h->ext.dev(), S.ext_out = h->ext.out;
    S.inj.ids = nullptr, S.ext.ids = nullptr;
    if (aniso) {  // the one-cell passes' arguments of the engine's own step (no density, no Q, FP32 state)
      AnisoBatchShot &A = ha[k];
      GradArgs &g = A.g;
      g.nx = d.nx, g.ny = d.ny, g.nz = d.nz, g.yseg = a.yseg, g.pml3d = h->c.pml3d;
      g.px = h->px, g.py = h->py, g.pz = h->pz;
      g.eps = h->eps, g.del = h->del, g.pjx = h->pjx, g.pjy = h->pjy;
      memcpy(g.c1x, h->c1x, sizeof g.c1x), memcpy(g.c1y, h->c1y, sizeof g.c1y), memcpy(g.c1z, h->c1z, sizeof g.c1z);
      g.pml = pml_dev(h);
      DivArgs &v = A.d;
      v.nx = d.nx, v.ny = d.ny, v.nz = d.nz, v.yseg = a.yseg, v.pml3d = h->c.pml3d;
      v.px = h->px, v.py = h->py, v.pz = h->pz, v.vel = h->vel;
      memcpy(v.c1x, h->c1x, sizeof v.c1x), memcpy(v.c1y, h->c1y, sizeof v.c1y), memcpy(v.c1z, h->c1z, sizeof v.c1z);
      v.pml = pml_dev(h);
      A.wa = S.wa, A.wb = S.wb;
      A.tiles_z = S.tiles_z, A.tiles_x = S.tiles_x, A.tiles_y = S.tiles_y, A.yseg = a.yseg;
    }
    start[k + 1] = start[k] + S.tiles_z * S.tiles_x * S.tiles_y;
    max_inj = std::max(max_inj, h->inj.ntr), max_ly = std::max(max_ly, h->inj.ly);
    max_ext = std::max(max_ext, h->ext.ntr);
  }
  if (n > b->cap) {
    cudaFree(b->d_shots), cudaFree(b->d_ashots), cudaFree(b->d_start);
    b->d_shots = nullptr, b->d_ashots = nullptr, b->d_start = nullptr, b->cap = 0;
    if (cudaMalloc(&b->d_shots, n * sizeof(IsoBatchShot)) != cudaSuccess ||
        (aniso && cudaMalloc(&b->d_ashots, n * sizeof(AnisoBatchShot)) != cudaSuccess) ||
        cudaMalloc(&b->d_start, (n + 1) * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      b->err = "batch table allocation failed";
      return RTM_ERR_NOMEM;
    }
    b->cap = n;
  }
  if (cudaMemcpyAsync(b->d_shots, hs.data(), n * sizeof(IsoBatchShot), cudaMemcpyHostToDevice, b->st) ||
      (aniso && cudaMemcpyAsync(b->d_ashots, ha.data(), n * sizeof(AnisoBatchShot), cudaMemcpyHostToDevice, b->st)) ||
      cudaMemcpyAsync(b->d_start, start.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, b->st)) {
    b->err = "batch table upload failed";
    return RTM_ERR_CUDA;
  }
  return RTM_OK;
}

// `count` steps of the shots in `order` (sorted by step count, descending:
// the active shots of step it are the prefix with nts > it), as CUDA graphs
// of up to 256 steps.  extract: ntratio > 0 gathers receivers every ntratio steps.
static int batch_run(rtm_batch *b, const std::vector<int> &order, const std::vector<int> &nts_sorted, int count,
                     int it_shift, int ntratio) {
  std::vector<int> start;
  int max_inj, max_ly, max_ext;
  TRY(batch_upload(b, order, start, max_inj, max_ly, max_ext));
  int num_sms = 0;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, b->device);
  const bool aniso = b->model != RTM_ISO;
  const int grid = (aniso ? aniso_batch_ctas_per_sm() : iso_batch_ctas_per_sm(b->tx, b->pml3d)) *
                   (num_sms > 0 ? num_sms : 148);
  const int n = (int)order.size();
  auto step = [&](int it) {
    int na = 0;
    while (na < n && nts_sorted[na] > it) na++;
    if (aniso) launch_aniso_fd8_batch(b->d_ashots, b->d_start, na, start[na], it, b->model, grid, b->st);
    else launch_iso_fd8_batch(b->d_shots, b->d_start, na, start[na], it, b->pml3d, b->tx, grid, b->st);
    launch_batch_inject(b->d_shots, na, max_inj, max_ly, it + it_shift, it, b->st);
    if (ntratio > 0 && it % ntratio == 0) launch_batch_extract(b->d_shots, na, max_ext, it / ntratio, it, b->st);
  };
  if (cudaEventRecord(b->ev0, b->st)) return RTM_ERR_CUDA;
  for (int s0 = 0; s0 < count; s0 += 256) {
    const int s1 = std::min(count, s0 + 256);
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal)) return RTM_ERR_CUDA;
    for (int it = s0; it < s1; it++) step(it);
    cudaError_t ec = cudaStreamEndCapture(b->st, &g);
    if (ec != cudaSuccess) {
      b->err = std::string("batch graph capture: ") + cudaGetErrorString(ec);
      cudaGetLastError();
      return RTM_ERR_CUDA;
    }
    cudaGraphExec_t ge = nullptr;
    cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      b->err = std::string("batch graph instantiate: ") + cudaGetErrorString(ei);
      cudaGetLastError();
      return RTM_ERR_CUDA;
    }
    cudaError_t el = cudaGraphLaunch(ge, b->st);
    cudaGraphExecDestroy(ge);
    if (el != cudaSuccess) {
      b->err = std::string("batch graph launch: ") + cudaGetErrorString(el);
      return RTM_ERR_CUDA;
    }
  }
  if (cudaEventRecord(b->ev1, b->st) || cudaEventSynchronize(b->ev1)) {
    b->err = std::string("batch loop: ") + cudaGetErrorString(cudaGetLastError());
    return RTM_ERR_CUDA;
  }
  cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
  return RTM_OK;
}
}  // namespace rtm

namespace rtm {
// The time-dependent propagation state, in a fixed order: the wavefields of
// the current step (w0, w1; FP16 state: the codes, the three slab scales and
// the two slab maxima in their current roles), the Q memory of both time
// levels (current first) and every PML memory array.  Saving and loading in
// the same order keeps the roles that the per-step swaps rotate.
static void state_pieces(Engine *h, std::vector<std::pair<void *, size_t>> &v) {
  const size_t n = (size_t)h->n, ny = (size_t)h->d.ny;
  if (h->f16) {
    v.push_back({h->h0, n * 2}), v.push_back({h->h1, n * 2});
    v.push_back({h->s0, ny * 4}), v.push_back({h->s1, ny * 4}), v.push_back({h->sn, ny * 4});
    v.push_back({h->m0, ny * 4}), v.push_back({h->m1, ny * 4});
  } else {
    v.push_back({h->w0, n * 4}), v.push_back({h->w1, n * 4});
  }
  if (h->c.use_q && h->wq[0]) {
    const size_t qb = (size_t)h->c.q_order * n * (h->c.q_bf16 ? 2 : 4);
    v.push_back({h->wq[h->iq0], qb}), v.push_back({h->wq[1 - h->iq0], qb});
  }
  for (int dim = 0; dim < 3; dim++)
    for (int sd = 0; sd < 2; sd++) {
      const PmlFace &F = h->pml.f[dim][sd];
      if (!F.w) continue;
      const long long plane = dim == DX ? (long long)h->d.ny * h->d.nz
                              : dim == DY ? (long long)h->d.nx * h->d.nz : (long long)h->d.nx * h->d.ny;
      for (int r = 0; r < 2; r++)
        for (int k = 0; k < 3; k++)
          if (F.q[r][k]) v.push_back({F.q[r][k], (size_t)plane * F.w * 4});
    }
}

// bytes of one snapshot slot of format fmt (256-byte multiples); the learned
// format with the handle's current FP16 fallback
static size_t slot_size(Engine *h, int fmt) {
  const size_t b = fmt == RTM_SNAP_FP32  ? (size_t)h->n * 4
                   : fmt == RTM_SNAP_C16 ? (size_t)(h->nxz + 2) * h->d.ny * 2
                   : fmt == RTM_SNAP_AE  ? ((size_t)ae_volume_blocks(h->d.nx, h->d.ny, h->d.nz) * 33 * 4 + 15) / 16 * 16 +
                                              (ae_fb_cap(h) ? ae_fallback_bytes(ae_fb_cap(h)) : 0)
                                         : (size_t)h->n * 2;
  return (b + 255) / 256 * 256;
}

static size_t state_size(Engine *h) {
  std::vector<std::pair<void *, size_t>> v;
  state_pieces(h, v);
  size_t b = 0;
  for (auto &p : v) b += (p.second + 255) / 256 * 256;
  return b;
}
}  // namespace rtm

extern "C" {

void rtm_config_default(rtm_config *c) {
  if (!c) return;
  memset(c, 0, sizeof *c);
  c->engine = RTM_ENGINE_FD8;
  c->model_type = RTM_ISO;
  c->q_order = 4;
  c->vmax = 4500.f;
  c->pml_eps = 1e-3f;
  c->pml3d = 1;
  c->pml3d_scaler = 0.3f;
  c->top_pml = 1;
}

const char *rtm_last_error(const rtm_handle *h) { return h ? h->err.c_str() : rtm::g_create_error.c_str(); }

int rtm_destroy(rtm_handle *h) {
  if (!h) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->st);
  for (void *p : h->allocs) cudaFree(p);
  h->allocs.clear();
  if (h->st_copy) cudaStreamSynchronize(h->st_copy);
  if (h->ic_plans) rtm::ic_plans_destroy(h->ic_plans);
  if (h->fft) rtm::fft_plans_destroy(h->fft);
  if (h->dbl_fft) rtm::fft_plans_destroy(h->dbl_fft);
  if (h->r2r) rtm::r2r_plans_destroy(h->r2r);
  if (h->host_snaps) cudaFreeHost(h->host_snaps);
  for (cudaEvent_t e : h->stage_ev)
    if (e) cudaEventDestroy(e);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->st_copy) cudaStreamDestroy(h->st_copy);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return RTM_OK;
}

int rtm_create(const rtm_dims *d, const rtm_config *c, rtm_handle **out) {
  using namespace rtm;
  if (!d || !c || !out) return RTM_ERR_ARG;
  *out = nullptr;
  if (d->nx < 9 || d->nz < 9 || d->ny < 1 || d->ny > 65535 || d->dx <= 0 || d->dy <= 0 || d->dz <= 0 || d->dt <= 0 || c->vmax <= 0 ||
      c->engine < 0 || c->engine > 6 || c->model_type < 1 || c->model_type > 3 || c->q_order < 1 || c->q_order > 8 ||
      c->pml_eps <= 0 || c->pml_eps >= 1) {
    g_create_error = "rtm_create: dimensions or configuration out of range";
    return RTM_ERR_ARG;
  }
  if (c->state_fp16 && (c->engine != RTM_ENGINE_FD8 || c->model_type < RTM_VTI || c->use_rho)) {
    g_create_error = "rtm_create: FP16 wavefield state is built for the FD8 VTI / TTI (+Q) path without density";
    return RTM_ERR_UNSUPPORTED;
  }
  rtm_handle *h = new rtm_handle();
  h->d = *d;
  h->c = *c;
  // FdEngine_r2c / _r2r and the Derivative path's Boundary damp only along
  // each derivative's own axis (bgprtm/FdEngine_r2c.cpp:240-243,
  // FdEngine_r2r.cpp:95-98, Boundary.cpp:153-213): no pml3d cross terms
  if (c->engine != RTM_ENGINE_FD8 && c->engine != RTM_ENGINE_CFD) h->c.pml3d = 0;
  h->n = (long long)d->nx * d->ny * d->nz;
  h->nxz = (long long)d->nx * d->nz;
  int rc = RTM_OK;
  auto fail = [&](int code) {
    g_create_error = "rtm_create: " + h->err;
    rtm_destroy(h);
    return code;
  };
  if (cudaGetDevice(&h->device) != cudaSuccess) {
    h->err = "no CUDA device";
    cudaGetLastError();
    return fail(RTM_ERR_CUDA);
  }
  // a blocking stream: its work waits for earlier legacy-stream work, so the
  // set-up uploads below (pageable cudaMemcpy, whose DMA may still be running
  // when the call returns) land before any kernel of the engine reads them
  if (cudaStreamCreate(&h->st) != cudaSuccess || cudaEventCreate(&h->ev0) != cudaSuccess ||
      cudaEventCreate(&h->ev1) != cudaSuccess) {
    h->err = "stream/event creation failed";
    cudaGetLastError();
    return fail(RTM_ERR_CUDA);
  }
  h->f16 = c->state_fp16 ? 1 : 0;
  if (h->f16) {
    if ((rc = h->alloc(h->h0, h->n)) || (rc = h->alloc(h->h1, h->n)) || (rc = h->alloc(h->s0, d->ny)) ||
        (rc = h->alloc(h->s1, d->ny)) || (rc = h->alloc(h->sn, d->ny)) || (rc = h->alloc(h->m0, d->ny)) ||
        (rc = h->alloc(h->m1, d->ny)))
      return fail(rc);
  } else if ((rc = h->alloc(h->w0, h->n)) || (rc = h->alloc(h->w1, h->n))) {
    return fail(rc);
  }
  if ((rc = h->alloc(h->vel, h->n)) || (rc = h->alloc(h->dflag, 1))) return fail(rc);
  const bool first_deriv = !h->lap_iso();
  if (first_deriv) {
    if ((rc = h->alloc(h->px, h->n)) || (rc = h->alloc(h->pz, h->n)) || (d->ny > 1 && (rc = h->alloc(h->py, h->n))))
      return fail(rc);
  }
  if (c->engine == RTM_ENGINE_R2C || c->engine == RTM_ENGINE_R2R || c->engine == RTM_ENGINE_FFTV ||
      c->engine == RTM_ENGINE_SINCOS) {
    if ((rc = h->alloc(h->scr, h->n)) || (rc = h->alloc(h->scr2, h->n))) return fail(rc);
    if ((c->engine == RTM_ENGINE_R2C || c->engine == RTM_ENGINE_FFTV) &&
        (rc = fft_plans_create(&h->fft, d->nx, d->ny, d->nz, d->dx, d->dy, d->dz, h->st, c->kernel_variant != 1,
                               h->dflag))) {
      h->err = "cuFFT plan set-up failed";
      return fail(rc);
    }
    if ((c->engine == RTM_ENGINE_R2R || c->engine == RTM_ENGINE_SINCOS) &&
        (rc = r2r_plans_create(&h->r2r, d->nx, d->ny, d->nz, d->dx, d->dy, d->dz, h->st, c->kernel_variant != 1,
                               h->dflag))) {
      h->err = "FFTWR2R line-matrix set-up failed";
      return fail(rc);
    }
  }
  if (c->engine == RTM_ENGINE_CFD || c->engine == RTM_ENGINE_CFDB) {
    if (cfd_init() != 0) {
      h->err = "compact-FD kernel set-up failed";
      cudaGetLastError();
      return fail(RTM_ERR_CUDA);
    }
    if ((rc = h->alloc(h->scr, h->n)) || (rc = h->alloc(h->scr2, h->n))) return fail(rc);
    const int nn[3] = {d->nx, d->ny, d->nz};
    const float dd[3] = {d->dx, d->dy, d->dz};
    for (int a = 0; a < 3; a++) {
      if (nn[a] < 16) {
        if (a == DY && nn[a] == 1) continue;
        h->err = "compact FD needs at least 16 cells per axis";
        return fail(RTM_ERR_ARG);
      }
      for (int s = 0; s < 2; s++) {
        std::vector<float> bm, bl, am, rd;
        cfd_plan(nn[a], dd[a], s + 1, bm, bl, am, &rd);
        std::vector<float> bu(4 * (size_t)nn[a]), lm(4 * (size_t)nn[a], 0.f);
        for (int i = 0; i < nn[a]; i++) {
          for (int k = 0; k < 4; k++) bu[(size_t)i * 4 + k] = bm[(size_t)i * 5 + 1 + k];
          for (int k = 0; k < 4; k++)
            if (i - 1 - k >= 0) lm[(size_t)i * 4 + k] = bl[(size_t)(i - 1 - k) * 4 + k];
        }
        float *dbu, *dbl, *dam, *drd, *dlm;
        if ((rc = h->alloc(dbu, bu.size())) || (rc = h->alloc(dbl, bl.size())) || (rc = h->alloc(dam, am.size())) ||
            (rc = h->alloc(drd, rd.size())) || (rc = h->alloc(dlm, lm.size())))
          return fail(rc);
        cudaMemcpy(dlm, lm.data(), lm.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dbu, bu.data(), bu.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dbl, bl.data(), bl.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dam, am.data(), am.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(drd, rd.data(), rd.size() * 4, cudaMemcpyHostToDevice);
        CfdPlanDev pd{nn[a], dbu, dbl, dam, drd, dlm, 1, 0, {0, 0, 0, 0}, {0, 0, 0, 0}, 0.f, {}};
        for (int k = 0; k < 60; k++) pd.a[k] = am[k];
        cfd_constant_run(nn[a], lm, bu, rd, pd);
        {  // segment layout and correction tables of the segment-parallel solve
          std::vector<float> hf, gb, hb;
          cfd_seg_layout(nn[a], pd.nseg, pd.seglen);
          cfd_seg_tables(nn[a], lm, bu, rd, pd.nseg, pd.seglen, hf, gb, hb);
          float *dhf, *dgb, *dhb;
          if ((rc = h->alloc(dhf, hf.size())) || (rc = h->alloc(dgb, gb.size())) || (rc = h->alloc(dhb, hb.size())))
            return fail(rc);
          cudaMemcpy(dhf, hf.data(), hf.size() * 4, cudaMemcpyHostToDevice);
          cudaMemcpy(dgb, gb.data(), gb.size() * 4, cudaMemcpyHostToDevice);
          cudaMemcpy(dhb, hb.data(), hb.size() * 4, cudaMemcpyHostToDevice);
          pd.hf = dhf, pd.gb = dgb, pd.hb = dhb;
        }
        h->cfd[a][s] = pd;
      }
    }
  }
  if (c->model_type >= RTM_VTI) {
    if ((rc = h->alloc(h->eps, h->n)) || (rc = h->alloc(h->del, h->n))) return fail(rc);
  }
  if (c->use_rho && (rc = h->alloc(h->rho, h->n))) return fail(rc);
  if (c->model_type == RTM_TTI) {
    if ((rc = h->alloc(h->pjx, h->n)) || (d->ny > 1 && (rc = h->alloc(h->pjy, h->n)))) return fail(rc);
  }
  if (c->use_q) {
    // BF16 memory variables take half the floats (rounded up to whole 16-byte rows)
    const size_t qn = c->q_bf16 ? ((size_t)c->q_order * h->n + 7) / 8 * 4 : (size_t)c->q_order * h->n;
    if ((rc = h->alloc(h->invq, h->n)) || (rc = h->alloc(h->wq[0], qn)) || (rc = h->alloc(h->wq[1], qn)))
      return fail(rc);
  }
  // FD tables (FdEngine_fd constructor + setJacob, rectangular grid, const order)
  double t1[5], t2[5];
  fd_weights(4, t1, t2);
  const float zpi = 1.0f / d->dz, zpi2 = zpi * zpi;
  const float dx2i = (float)(1.0 / (double)(d->dx * d->dx)), dy2i = (float)(1.0 / (double)(d->dy * d->dy));
  const float dxi = 1.0f / d->dx, dyi = 1.0f / d->dy;
  for (int m = 0; m < 5; m++) {
    const float c2 = (float)t2[m], c1 = m ? (float)t1[m] : 0.f;
    h->c2z[m] = zpi2 * c2, h->c2x[m] = c2 * dx2i, h->c2y[m] = c2 * dy2i;
    h->c1z[m] = zpi * c1, h->c1x[m] = c1 * dxi, h->c1y[m] = c1 * dyi;
  }
  if ((rc = setup_pml(h))) return fail(rc);
  // imaging-condition tapers (edge tapers of the decode, depth taper default off)
  std::vector<float> tx, ty, tz, one;
  edge_taper(d->nx, 20, tx), edge_taper(d->ny, 20, ty), edge_taper(d->nz, 10, tz);
  if ((rc = h->alloc(h->ex, d->nx)) || (rc = h->alloc(h->ey, d->ny)) || (rc = h->alloc(h->ez, d->nz)) ||
      (rc = h->alloc(h->one_x, d->nx)) || (rc = h->alloc(h->one_y, d->ny)) || (rc = h->alloc(h->one_z, d->nz)) ||
      (rc = h->alloc(h->taper_z, d->nz)))
    return fail(rc);
  cudaMemcpy(h->ex, tx.data(), 4 * d->nx, cudaMemcpyHostToDevice);
  cudaMemcpy(h->ey, ty.data(), 4 * d->ny, cudaMemcpyHostToDevice);
  cudaMemcpy(h->ez, tz.data(), 4 * d->nz, cudaMemcpyHostToDevice);
  one.assign(std::max(std::max(d->nx, d->ny), d->nz), 1.0f);
  cudaMemcpy(h->one_x, one.data(), 4 * d->nx, cudaMemcpyHostToDevice);
  cudaMemcpy(h->one_y, one.data(), 4 * d->ny, cudaMemcpyHostToDevice);
  cudaMemcpy(h->one_z, one.data(), 4 * d->nz, cudaMemcpyHostToDevice);
  cudaMemcpy(h->taper_z, one.data(), 4 * d->nz, cudaMemcpyHostToDevice);
  choose_shape(h);
  h->use_tma = (c->kernel_variant == 0 || c->kernel_variant == 2) && tma_supported(d->nz) && iso_tma_init();
  if (h->lap_iso() && d->nz % 4 == 0 &&
      (c->kernel_variant == 0 || c->kernel_variant == 3 || c->kernel_variant == 4)) {
    h->iso4 = c->kernel_variant != 4 && tma_supported(d->nz) && iso_tma4_init() ? 2 : 1;
    h->v4_yseg = yseg_iso4(h);
    if (h->iso4 == 2 && (rc = iso4_tiles(h))) return fail(rc);
  }
  if (c->engine == RTM_ENGINE_FD8 && !h->lap_iso() && (rc = fd8_tiles(h))) return fail(rc);
  // the 4-cell passes carry no density term: a density model runs the one-cell passes
  if (c->engine == RTM_ENGINE_FD8 && !h->lap_iso() && !c->use_rho && !c->state_fp16 && d->nz % 4 == 0 &&
      (c->kernel_variant == 0 || c->kernel_variant == 3 || c->kernel_variant == 7) && tma_supported(d->nz) &&
      aniso4_init()) {
    h->aniso4 = 1;
    h->an4_yseg = yseg_an4(h);
    if ((rc = an4_tiles(h))) return fail(rc);
  }
  // BF16 rows of the Q-memory tensor maps need nz % 8 == 0 (16-byte strides)
  h->qring_ok = c->kernel_variant != 7 && (!c->q_bf16 || d->nz % 8 == 0);
  h->cfd_tma = (c->engine == RTM_ENGINE_CFD || c->engine == RTM_ENGINE_CFDB) && tma_supported(d->nz);
  // compact FD: the split pipeline (line solves + pointwise epilogues) with TMA
  // x / y tiles by default (register-streamed lines without tensor maps), the
  // faster form on the 512x512x400 workload; 5 / 1 / 2 force its streamed /
  // plain / TMA x / y lines.  On 3-D grids whose lines fit a tile, 8 selects
  // the segment-parallel fused pipeline (TMA tile loads where the tensor maps
  // can be made) and 6 its plain-load form; the autotuner tries both forms.
  h->cfd_seg_ok = c->engine == RTM_ENGINE_CFD && d->ny > 1 && d->nx <= cfd_seg_max_n(DX) &&
                  d->ny <= cfd_seg_max_n(DY) && d->nz <= cfd_seg_max_n(DZ) && cfd_seg_init() == 0;
  h->cfd_zfuse = c->kernel_variant == 9;
  h->cfd_pipe = c->kernel_variant == 10;
  if (c->kernel_variant == 0 || c->kernel_variant == 9 || c->kernel_variant == 10) h->cfd_xy = h->cfd_tma ? 1 : 0;
  else if (c->kernel_variant == 5) h->cfd_xy = 0;
  else if (c->kernel_variant == 6 && h->cfd_seg_ok) h->cfd_xy = 4;
  else if (c->kernel_variant == 8 && h->cfd_seg_ok) h->cfd_xy = h->cfd_tma ? 3 : 4;
  else h->cfd_xy = c->kernel_variant == 2 && h->cfd_tma ? 1 : 2;
  cudaGetLastError();
  CK(cudaMemset(h->dflag, 0, sizeof(int)));
  if ((rc = zero_state(h))) return fail(rc);
  if (cudaStreamSynchronize(h->st) != cudaSuccess) {
    h->err = "initialisation failed";
    cudaGetLastError();
    return fail(RTM_ERR_CUDA);
  }
  *out = h;
  return RTM_OK;
}

int rtm_set_q_coeffs(rtm_handle *h, float cq0, const float *cq, const float *wq) {
  if (!h || !cq || !wq) return RTM_ERR_ARG;
  if (!h->c.use_q) {
    h->err = "use_q is off";
    return RTM_ERR_STATE;
  }
  h->cq0 = cq0;
  h->cqsum = 0.f;
  for (int l = 0; l < h->c.q_order; l++) h->cq[l] = cq[l], h->cwq[l] = wq[l], h->cqsum += cq[l];
  h->q_set = 1;
  return RTM_OK;
}

int rtm_set_model(rtm_handle *h, const float *vel, const float *rho, const float *eps, const float *del,
                  const float *pjx, const float *pjy, const float *invq) {
  using namespace rtm;
  if (!h || !vel) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  const int mt = h->c.model_type;
  if ((mt >= RTM_VTI && (!eps || !del)) || (mt == RTM_TTI && (!pjx || (h->d.ny > 1 && !pjy))) ||
      (h->c.use_q && !invq)) {
    h->err = "model arrays required by the model type are missing";
    return RTM_ERR_ARG;
  }
  if (!h->c.use_rho != !rho) {
    h->err = h->c.use_rho ? "use_rho is set: rtm_set_model needs the density volume"
                          : "a density volume needs use_rho in the configuration of rtm_create";
    return RTM_ERR_ARG;
  }
  if (rho)
    for (long long i = 0; i < h->n; i++)
      if (!std::isfinite(rho[i]) || rho[i] <= 0.f) {
        h->err = "density not finite or not positive at cell " + std::to_string(i);
        return RTM_ERR_NONFINITE;
      }
  if (h->c.use_q && !h->q_set) {
    h->err = "rtm_set_q_coeffs must precede rtm_set_model when use_q";
    return RTM_ERR_STATE;
  }
  for (long long i = 0; i < h->n; i++)
    if (!std::isfinite(vel[i]) || vel[i] <= 0.f) {
      h->err = "velocity not finite or not positive at cell " + std::to_string(i);
      return RTM_ERR_NONFINITE;
    }
  const size_t bytes = (size_t)h->n * 4;
  {
    float vmx = 0.f;
    for (long long i = 0; i < h->n; i++) vmx = std::max(vmx, vel[i]);
    h->vel2max = (vmx * h->d.dt) * (vmx * h->d.dt);
  }
  CK(cudaMemcpyAsync(h->vel, vel, bytes, cudaMemcpyHostToDevice, h->st));
  if (mt >= RTM_VTI) {
    CK(cudaMemcpyAsync(h->eps, eps, bytes, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->del, del, bytes, cudaMemcpyHostToDevice, h->st));
  }
  if (mt == RTM_TTI) {
    CK(cudaMemcpyAsync(h->pjx, pjx, bytes, cudaMemcpyHostToDevice, h->st));
    if (h->d.ny > 1) CK(cudaMemcpyAsync(h->pjy, pjy, bytes, cudaMemcpyHostToDevice, h->st));
  }
  if (h->c.use_q) CK(cudaMemcpyAsync(h->invq, invq, bytes, cudaMemcpyHostToDevice, h->st));
  if (rho) CK(cudaMemcpyAsync(h->rho, rho, bytes, cudaMemcpyHostToDevice, h->st));
  launch_vel2(h->vel, h->invq, h->n, h->d.dt * h->d.dt, h->cq0, h->c.use_q, h->st);
  TRY(check_launch(h, "vel2"));
  CK(cudaStreamSynchronize(h->st));
  h->model_set = 1;
  return RTM_OK;
}

int rtm_reset(rtm_handle *h) {
  if (!h) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  TRY(rtm::zero_state(h));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_kernel(rtm_handle *h) {
  TRY(rtm::ready(h));
  if (h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  TRY(rtm::step_kernel(h, 0, rtm::io_none()));
  CK(cudaStreamSynchronize(h->st));
  return rtm::check_flag(h);
}

int rtm_update2nd(rtm_handle *h) {
  TRY(rtm::ready(h));
  if (h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  rtm::QDev q = rtm::q_dev(h);
  rtm::launch_update2nd(h->w0, h->w1, h->c.use_q ? &q : nullptr, h->n, h->st);
  TRY(rtm::check_launch(h, "update2nd"));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_swap(rtm_handle *h) {
  if (!h) return RTM_ERR_ARG;
  if (h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  rtm::do_swap(h);
  return RTM_OK;
}

int rtm_spread_coeffs(int n, float x, float k1, float k2, int *nlimit, int dipole, int ntaper, float *coeff, int *off) {
  if (!nlimit || !coeff || !off || n < 1 || !(k1 > 0.f) || k1 > k2 || k2 > 0.5f || !std::isfinite(x)) return RTM_ERR_ARG;
  if (n > 1 && (x < 0.f || x > (float)(n - 1))) return RTM_ERR_ARG;
  *off = rtm::spread_coeffs(n, x, k1, k2, nlimit, dipole, ntaper, coeff);
  return RTM_OK;
}

int rtm_r2r_line_matrix(int n, float d, int isign, float *D) {
  if (!D || n < 2 || n > 65536 || !(d > 0.f) || (isign != 1 && isign != -1)) return RTM_ERR_ARG;
  std::vector<float> m;
  rtm::r2r_line_matrix(n, d, isign, m);
  std::memcpy(D, m.data(), m.size() * 4);
  return RTM_OK;
}

int rtm_set_injection(rtm_handle *h, int ntr, int lx, int ly, int lz, const int *off3, const int *len3, const float *kx,
                      const float *ky, const float *kz, const float *traces, int nt, float scaler) {
  if (!h || ntr < 0 || (ntr > 0 && (!off3 || !len3 || !kx || !ky || !kz || !traces || nt <= 0 || lx < 1 || ly < 1 ||
                                   lz < 1)))
    return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  if (ntr > 0) {  // the largest value one injection can add: floor of the FP16 state's scales
    float tm = 0.f, km[3] = {0.f, 0.f, 0.f};
    for (long long i = 0; i < (long long)ntr * nt; i++) tm = std::max(tm, std::fabs(traces[i]));
    const float *kk[3] = {kx, ky, kz};
    const int ll[3] = {lx, ly, lz};
    for (int a = 0; a < 3; a++)
      for (long long i = 0; i < (long long)ntr * ll[a]; i++) km[a] = std::max(km[a], std::fabs(kk[a][i]));
    const float amp = tm * std::fabs(scaler) * km[0] * km[1] * km[2] * (h->vel2max > 0.f ? h->vel2max : 1.f);
    if (amp > 0.f && std::isfinite(amp)) h->f16_floor = amp;
  }
  return rtm::upload_traces(h, h->inj, ntr, lx, ly, lz, off3, len3, kx, ky, kz, traces, nt, scaler, false);
}

int rtm_set_extraction(rtm_handle *h, int ntr, int lx, int ly, int lz, const int *off3, const int *len3, const float *kx,
                       const float *ky, const float *kz, int nt_out) {
  if (!h || ntr < 0 ||
      (ntr > 0 && (!off3 || !len3 || !kx || !ky || !kz || nt_out <= 0 || lx < 1 || ly < 1 || lz < 1)))
    return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  return rtm::upload_traces(h, h->ext, ntr, lx, ly, lz, off3, len3, kx, ky, kz, nullptr, nt_out, 1.f, true);
}

int rtm_inject(rtm_handle *h, int it) {
  TRY(rtm::ready(h));
  if (h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  TRY(rtm::do_inject(h, it));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_extract(rtm_handle *h, int jt) {
  TRY(rtm::ready(h));
  if (h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  TRY(rtm::do_extract(h, jt));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_get_traces(rtm_handle *h, float *dst) {
  if (!h || !dst) return RTM_ERR_ARG;
  if (!h->ext.out) {
    h->err = "no extraction set";
    return RTM_ERR_STATE;
  }
  cudaSetDevice(h->device);
  CK(cudaMemcpyAsync(dst, h->ext.out, 4 * (size_t)h->ext.ntr * h->ext.nt, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_snapshot_setup(rtm_handle *h, int fmt, int nslots) {
  if (!h || nslots < 0 || fmt < RTM_SNAP_FP32 || fmt > RTM_SNAP_AE) return RTM_ERR_ARG;
  if (fmt == RTM_SNAP_AE && !h->ae) {
    h->err = "RTM_SNAP_AE needs rtm_set_compressor first";
    return RTM_ERR_STATE;
  }
  cudaSetDevice(h->device);
  if (h->st_copy) cudaStreamSynchronize(h->st_copy);
  if (h->host_snaps) cudaFreeHost(h->host_snaps);
  h->host_snaps = nullptr, h->nstage = 0;
  h->release(h->snaps), h->release(h->slabs), h->release(h->ae_scratch);
  h->snaps = nullptr, h->slabs = nullptr, h->ae_scratch = nullptr;
  h->snap_fmt = fmt, h->nslots = nslots, h->slot0 = 0;
  h->slot_bytes = rtm::slot_size(h, fmt);
  h->stored.assign(nslots, 0);
  if (!nslots) return RTM_OK;
  TRY(h->alloc(h->snaps, h->slot_bytes * nslots));
  if (fmt == RTM_SNAP_C16 || fmt == RTM_SNAP_FP16S) TRY(h->alloc(h->slabs, (size_t)nslots * h->d.ny));
  if (fmt == RTM_SNAP_AE) TRY(h->alloc(h->ae_scratch, h->n));
  return RTM_OK;
}


int rtm_checkpoint_setup(rtm_handle *h, int nckpt, size_t *bytes_each) {
  if (!h || nckpt < 0) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  CK(cudaStreamSynchronize(h->st));
  h->release(h->ckpts);
  h->ckpts = nullptr, h->nckpt = 0;
  h->ckpt_bytes = rtm::state_size(h);
  if (bytes_each) *bytes_each = h->ckpt_bytes;
  if (!nckpt) return RTM_OK;
  TRY(h->alloc(h->ckpts, h->ckpt_bytes * (size_t)nckpt));
  h->nckpt = nckpt;
  return RTM_OK;
}

static int checkpoint_copy(rtm_handle *h, int k, bool save) {
  if (!h || k < 0 || k >= h->nckpt) return RTM_ERR_ARG;
  TRY(rtm::ready(h));
  std::vector<std::pair<void *, size_t>> v;
  rtm::state_pieces(h, v);
  char *base = h->ckpts + (size_t)k * h->ckpt_bytes;
  for (auto &p : v) {
    if (save) CK(cudaMemcpyAsync(base, p.first, p.second, cudaMemcpyDeviceToDevice, h->st));
    else CK(cudaMemcpyAsync(p.first, base, p.second, cudaMemcpyDeviceToDevice, h->st));
    base += (p.second + 255) / 256 * 256;
  }
  return RTM_OK;
}

int rtm_checkpoint_save(rtm_handle *h, int k) { return checkpoint_copy(h, k, true); }
int rtm_checkpoint_load(rtm_handle *h, int k) { return checkpoint_copy(h, k, false); }

int rtm_snapshot_window(rtm_handle *h, int first) {
  if (!h) return RTM_ERR_ARG;
  h->slot0 = first;
  std::fill(h->stored.begin(), h->stored.end(), 0);
  return RTM_OK;
}

int rtm_snapshot_slot_bytes(rtm_handle *h, int fmt, size_t *bytes) {
  if (!h || !bytes || fmt < RTM_SNAP_FP32 || fmt > RTM_SNAP_AE) return RTM_ERR_ARG;
  *bytes = rtm::slot_size(h, fmt);
  return RTM_OK;
}

int rtm_set_compressor(rtm_handle *h, rtm_ae *a) {
  if (!h) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  h->ae = a;
  if (a && rtm::ae_prepare(a) != RTM_OK) {
    h->err = "compressor workspace allocation failed";
    return RTM_ERR_NOMEM;
  }
  return RTM_OK;
}

int rtm_set_compressor_fallback(rtm_handle *h, float tau, float max_fraction) {
  if (!h || tau < 0.f || tau >= 1.f || max_fraction < 0.f || max_fraction > 1.f) return RTM_ERR_ARG;
  h->ae_fb_tau = tau, h->ae_fb_frac = max_fraction;
  if (h->snap_fmt == RTM_SNAP_AE && h->nslots) TRY(rtm_snapshot_setup(h, RTM_SNAP_AE, h->nslots));  // new slot size
  return RTM_OK;
}

int rtm_snapshot_offload(rtm_handle *h, int nstage) {
  if (!h || nstage < 0 || nstage == 1 || nstage > 8) return RTM_ERR_ARG;
  if (nstage && h->snap_fmt == RTM_SNAP_AE) {
    h->err = "snapshot offload stores the FP32 / COMPRESS_16 / FP16 formats";
    return RTM_ERR_UNSUPPORTED;
  }
  cudaSetDevice(h->device);
  if (!h->st_copy) {
    if (cudaStreamCreateWithFlags(&h->st_copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess)
      return rtm::cuda_fail(cudaGetLastError(), "snapshot offload streams", h);
    for (cudaEvent_t &e : h->stage_ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        return rtm::cuda_fail(cudaGetLastError(), "snapshot offload events", h);
  }
  const int fmt = h->snap_fmt, nslots = h->nslots;
  TRY(rtm_snapshot_setup(h, fmt, nslots));  // drops any previous slots and their contents
  if (!nstage || !nslots) return RTM_OK;
  h->release(h->snaps);
  h->snaps = nullptr;
  TRY(h->alloc(h->snaps, h->slot_bytes * nstage));
  if (cudaHostAlloc((void **)&h->host_snaps, h->slot_bytes * nslots, cudaHostAllocDefault) != cudaSuccess) {
    h->host_snaps = nullptr;
    h->err = "cudaHostAlloc of " + std::to_string(h->slot_bytes * nslots) + " bytes failed";
    cudaGetLastError();
    return RTM_ERR_NOMEM;
  }
  h->nstage = nstage;
  for (int k = 0; k < 8; k++) h->stage_slot[k] = -1, h->stage_wait[k] = false;
  return RTM_OK;
}

int rtm_snapshot_store(rtm_handle *h, int slot) {
  TRY(rtm::ready(h));
  if (h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  if (slot < 0 || slot >= h->nslots) return RTM_ERR_ARG;
  if (h->nstage) TRY(rtm::stage_ready(h, slot));
  if (h->snap_fmt == RTM_SNAP_AE) {
    TRY(rtm::ae_store(h, slot, h->w0));
  } else {
    TRY(rtm::snap_prepare(h, slot));
    rtm::launch_fused_io(rtm::io_store(h, slot), h->w0, h->d.nx, h->d.ny, h->d.nz, h->st);
    TRY(rtm::check_launch(h, "snapshot_store"));
  }
  if (h->nstage) {
    TRY(rtm::offload_d2h(h, slot));
    TRY(rtm::stage_join(h));
  }
  h->stored[slot] = 1;
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_snapshot_load(rtm_handle *h, int slot, float *dst) {
  if (!h || !dst || slot < 0 || slot >= h->nslots) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->nstage) {
    TRY(rtm::stage_join(h));
    TRY(rtm::offload_h2d(h, slot));
    TRY(rtm::stage_ready(h, slot));
  }
  float *tmp = nullptr;
  TRY(h->alloc(tmp, h->n));
  int rc;
  if (h->snap_fmt == RTM_SNAP_AE) {
    rc = rtm::ae_load(h, slot, tmp);
  } else {
    rtm::launch_snap_decode(rtm::slot_dev(h, slot), tmp, h->ex, h->ey, h->ez, h->d.nx, h->d.ny, h->d.nz, h->st);
    rc = rtm::check_launch(h, "snapshot_load");
  }
  if (rc == RTM_OK) {
    cudaError_t e = cudaMemcpyAsync(dst, tmp, 4 * (size_t)h->n, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) rc = rtm::cuda_fail(e, "snapshot_load copy", h);
  }
  h->release(tmp);
  return rc;
}

int rtm_image_setup(rtm_handle *h, int ntaper_t, int ntaper_z, int edge) {
  if (!h || ntaper_t < 0 || ntaper_z < 0 || ntaper_z > h->d.nz) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->image) {
    TRY(h->alloc(h->image, h->n));
    TRY(h->alloc(h->comp, h->n));
  }
  CK(cudaMemsetAsync(h->image, 0, 4 * (size_t)h->n, h->st));
  CK(cudaMemsetAsync(h->comp, 0, 4 * (size_t)h->n, h->st));
  if (h->dbl) {
    CK(cudaMemsetAsync(h->dbl_img, 0, 4 * (size_t)h->n * h->dmap.nloop, h->st));
    CK(cudaMemsetAsync(h->dbl_comp, 0, 4 * (size_t)h->n * h->dmap.nloop, h->st));
  }
  // ImagingCondition::calTapes (bgprtm/ImagingCondition.cpp:180-198)
  h->taper_t.resize(ntaper_t);
  for (int i = 0; i < ntaper_t; i++) h->taper_t[i] = 0.5f * (1.0f - cosf((float)M_PI * float(i) / float(ntaper_t)));
  std::vector<float> tz(h->d.nz, 1.0f);
  for (int i = 0; i < ntaper_z; i++) tz[i] = 0.5f * (1.0f - cosf((float)M_PI * float(i) / float(ntaper_z)));
  CK(cudaMemcpyAsync(h->taper_z, tz.data(), 4 * h->d.nz, cudaMemcpyHostToDevice, h->st));
  h->ic_edge = edge ? 1 : 0;
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_image_condition(rtm_handle *h, int option) {
  if (!h || (option != RTM_IC_IMAGE1 && option != RTM_IC_INVERSION)) return RTM_ERR_ARG;
  if (option == RTM_IC_INVERSION && h->dbl) {
    h->err = "the double-grid imaging condition runs with RTM_IC_IMAGE1 only";
    return RTM_ERR_UNSUPPORTED;
  }
  cudaSetDevice(h->device);
  if (option == RTM_IC_INVERSION && !h->ic_plans) {
    h->ic_plans = rtm::ic_plans_create(h->d.nx, h->d.ny, h->d.nz);
    if (!h->ic_plans) {
      h->err = "cuFFT plan creation failed";
      return RTM_ERR_CUDA;
    }
    const long long nc = rtm::ic_spectrum_floats(h->d.nx, h->d.ny, h->d.nz);
    TRY(h->alloc(h->icS, h->n));
    TRY(h->alloc(h->icR, h->n));
    TRY(h->alloc(h->icDs, h->n));
    TRY(h->alloc(h->icDr, h->n));
    TRY(h->alloc(h->icSh, (size_t)nc));
    TRY(h->alloc(h->icRh, (size_t)nc));
    TRY(h->alloc(h->icTh, (size_t)nc));
  }
  h->ic_opt = option;
  return RTM_OK;
}

int rtm_image_double(rtm_handle *h, int ndbl_z, int ndbl_x, int ndbl_y, float high_z, float high_xy) {
  if (!h) return RTM_ERR_ARG;
  auto in12 = [](int v) { return v == 1 || v == 2; };
  if (!in12(ndbl_z) || !in12(ndbl_x) || !in12(ndbl_y) || !(high_z >= 0.f && high_z < 1.f) ||
      !(high_xy >= 0.f && high_xy < 1.f))
    return RTM_ERR_ARG;
  const rtm_dims &d = h->d;
  const bool on = ndbl_z == 2 || ndbl_x == 2 || ndbl_y == 2;
  if (on) {
    // ImagingCorrelator (bgprtm/ImagingCorrelator.cpp:57-74) needs z doubled whenever x or y
    // is; its interleave of a 3-D grid is complete only with all three doubled
    // (interleave2d moves one xz plane), and x / y are never doubled on a 1-cell axis
    const bool ok = ndbl_z == 2 && (d.nx > 1 || ndbl_x == 1) &&
                    (d.ny == 1 ? ndbl_y == 1 : (d.nx > 1 && ndbl_x == 2 && ndbl_y == 2));
    if (!ok) {
      h->err = "double-grid imaging: supported factors are (z, x, y) = (2, 1, 1) or (2, 2, 1) on 2-D grids and "
               "(2, 2, 2) on 3-D grids";
      return RTM_ERR_ARG;
    }
    if (h->ic_opt == RTM_IC_INVERSION) {
      h->err = "the double-grid imaging condition runs with RTM_IC_IMAGE1 only";
      return RTM_ERR_UNSUPPORTED;
    }
  }
  cudaSetDevice(h->device);
  CK(cudaStreamSynchronize(h->st));
  // release an earlier set-up
  for (float *&p : h->dblS) h->release(p), p = nullptr;
  for (float *&p : h->dblR) h->release(p), p = nullptr;
  h->release(h->dbl_img), h->release(h->dbl_comp);
  h->dbl_img = h->dbl_comp = nullptr;
  if (h->dbl_fft) rtm::fft_plans_destroy(h->dbl_fft), h->dbl_fft = nullptr;
  h->dbl = 0;
  if (!on) return RTM_OK;
  // copy slots as ImagingCorrelator: ivz = 1, ivx = 2, ivy = 3, ivzx = 4, ivzy = 5, ivxy = 6,
  // ivzxy = 7, renumbered when an axis is not doubled
  int ivz = 1, ivx = 2, ivy = 3, ivzx = 4, ivzy = 5, ivxy = 6, ivzxy = 7;
  if (ndbl_y == 1) {
    if (ndbl_x == 1) ivz = 1;
    else ivz = 1, ivx = 2, ivzx = 3;
    ivy = ivxy = ivzy = ivzxy = 0;
  }
  if (ndbl_x == 1) ivx = ivxy = ivzx = ivzxy = 0;
  rtm::DblMap m{};
  m.dz = ndbl_z, m.dx = ndbl_x, m.dy = ndbl_y;
  m.nloop = ivzxy ? 8 : ivzx ? 4 : 2;
  const int iv[7] = {ivz, ivx, ivy, ivzx, ivzy, ivxy, ivzxy};
  for (int k = 0; k < 7; k++) m.iv[k] = iv[k];
  // point class c = 4 (y odd) + 2 (x odd) + (z odd)
  m.slot[0] = 0, m.slot[1] = ivz, m.slot[2] = ivx, m.slot[3] = ivzx, m.slot[4] = ivy, m.slot[5] = ivzy,
  m.slot[6] = ivxy, m.slot[7] = ivzxy;
  const int rc = rtm::fft_plans_create(&h->dbl_fft, d.nx, d.ny, d.nz, (float)d.dx, (float)d.dy, (float)d.dz, h->st);
  if (rc != RTM_OK) {
    h->err = "double-grid imaging: line-FFT plan creation failed";
    return rc;
  }
  for (int i = 0; i < m.nloop; i++) {
    TRY(h->alloc(h->dblS[i], h->n));
    TRY(h->alloc(h->dblR[i], h->n));
  }
  TRY(h->alloc(h->dbl_img, (size_t)h->n * m.nloop));
  TRY(h->alloc(h->dbl_comp, (size_t)h->n * m.nloop));
  CK(cudaMemsetAsync(h->dbl_img, 0, 4 * (size_t)h->n * m.nloop, h->st));
  CK(cudaMemsetAsync(h->dbl_comp, 0, 4 * (size_t)h->n * m.nloop, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->dmap = m;
  h->dbl_hz = high_z, h->dbl_hxy = high_xy;
  h->dbl = 1;
  return RTM_OK;
}

// the doubled-grid image or illumination into host memory (dst: n * nloop floats)
static int get_double(Engine *h, bool illum, float *dst) {
  if (!h || !dst) return RTM_ERR_ARG;
  if (!h->dbl || (illum && !h->illum)) {
    h->err = illum ? "no double-grid imaging set-up or no illumination" : "no double-grid imaging set-up";
    return RTM_ERR_STATE;
  }
  cudaSetDevice(h->device);
  const size_t n2 = (size_t)h->n * h->dmap.nloop;
  float *tmp = nullptr;
  TRY(h->alloc(tmp, n2));
  if (illum) rtm::launch_dbl_illum(h->illum, tmp, h->dmap, h->d.nx, h->d.ny, h->d.nz, h->st);
  else rtm::launch_dbl_interleave(h->dbl_img, tmp, h->dmap, h->d.nx, h->d.ny, h->d.nz, h->st);
  int rc = rtm::check_launch(h, illum ? "dbl_illum" : "dbl_interleave");
  if (rc == RTM_OK) {
    cudaError_t e = cudaMemcpyAsync(dst, tmp, 4 * n2, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) rc = rtm::cuda_fail(e, "double-grid readout", h);
  }
  h->release(tmp);
  return rc;
}
int rtm_get_image_double(rtm_handle *h, float *dst) { return get_double(h, false, dst); }
int rtm_get_illum_double(rtm_handle *h, float *dst) { return get_double(h, true, dst); }

int rtm_illum_setup(rtm_handle *h, int on) {
  if (!h) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  if (on && !h->illum) TRY(h->alloc(h->illum, h->n));
  if (h->illum) CK(cudaMemsetAsync(h->illum, 0, 4 * (size_t)h->n, h->st));
  h->illum_on = on ? 1 : 0;
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_illum_compensate(rtm_handle *h, int smooth_xy, int smooth_z, float amp_damping, float damp_weight) {
  if (!h || !h->illum || !h->image || smooth_xy < 0 || smooth_z < 0) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  float *tmp = nullptr;
  double *dsum = nullptr;
  int rc = h->alloc(tmp, h->n);
  if (rc == RTM_OK) rc = h->alloc(dsum, 1);
  if (rc == RTM_OK) {
    rtm::launch_illum_compensate(h->illum, tmp, h->image, dsum, h->d.nx, h->d.ny, h->d.nz, smooth_xy > 0 || smooth_z > 0,
                                 smooth_xy, smooth_z, amp_damping, damp_weight, h->st);
    rc = rtm::check_launch(h, "illum_compensate");
    const cudaError_t e = cudaStreamSynchronize(h->st);
    if (rc == RTM_OK && e != cudaSuccess) rc = rtm::cuda_fail(e, "illum_compensate", h);
  }
  h->release(tmp), h->release(dsum);
  return rc;
}

int rtm_image_accumulate(rtm_handle *h, int slot) {
  if (h && h->f16) {
    h->err = "the stepwise KernelCPU-seam calls do not run on FP16 wavefield state; use the loop drivers";
    return RTM_ERR_UNSUPPORTED;
  }
  TRY(rtm::ready(h));
  if (slot < 0 || slot >= h->nslots || !h->image) return RTM_ERR_ARG;
  if (!h->stored[slot]) return RTM_OK;
  if (h->nstage) {
    TRY(rtm::offload_h2d(h, slot));
    TRY(rtm::stage_ready(h, slot));
  }
  if (h->ic_opt == RTM_IC_INVERSION || h->dbl) {
    if (h->snap_fmt == RTM_SNAP_AE) TRY(rtm::ae_load(h, slot, h->ae_scratch));
    if (h->dbl) TRY(rtm::ic_double_explicit(h, slot, h->w0));
    else TRY(rtm::ic_explicit(h, slot, h->w0));
  } else {
    rtm::launch_fused_io(rtm::io_image(h, slot), h->w0, h->d.nx, h->d.ny, h->d.nz, h->st);
    TRY(rtm::check_launch(h, "image_accumulate"));
  }
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_modelling(rtm_handle *h, int nts, int it_shift, int ntratio) {
  TRY(rtm::ready(h));
  if (nts < 0 || ntratio < 1) return RTM_ERR_ARG;
  const int mode = h->c.use_q ? 2 : 1;
  return rtm::run_graphs(h, nts, [&](int it) {
    TRY(rtm::step_kernel(h, mode, rtm::io_none()));
    TRY(rtm::do_inject(h, it + it_shift));
    if (it % ntratio == 0) TRY(rtm::do_extract(h, it / ntratio));
    rtm::do_swap(h);
    return (int)RTM_OK;
  });
}

int rtm_migration(rtm_handle *h, int dir, int it_begin, int it_end, int it_shift, int interval) {
  TRY(rtm::ready(h));
  if ((dir != RTM_FORWARD && dir != RTM_BACKWARD) || interval < 1) return RTM_ERR_ARG;
  if (dir == RTM_BACKWARD && !h->image) {
    h->err = "rtm_image_setup must precede a backward migration";
    return RTM_ERR_STATE;
  }
  const int inc = dir == RTM_FORWARD ? 1 : -1;
  const int count = dir == RTM_FORWARD ? it_end - it_begin : it_begin - it_end;
  if (count < 0) return RTM_ERR_ARG;
  const int mode = h->c.use_q ? 2 : 1;
  rtm::FusedIo pending = rtm::io_none();
  int pending_slot = -1;  // slot the pending store writes (offload: copied to the host after it)
  const bool off = h->nstage > 0;
  int rc = rtm::run_graphs(h, count, [&](int s) {
    const int it = it_begin + s * inc;
    TRY(rtm::step_kernel(h, mode, pending));
    if (off && pending.store) TRY(rtm::offload_d2h(h, pending_slot));
    pending = rtm::io_none(), pending_slot = -1;
    TRY(rtm::do_inject(h, it + it_shift * inc));
    if (it % interval == 0) {
      const int slot = it / interval - h->slot0;
      if (slot >= 0 && slot < h->nslots) {
        if (dir == RTM_FORWARD) {
          if (h->snap_fmt == RTM_SNAP_AE) {
            TRY(rtm::ae_store(h, slot, h->f16 ? rtm::f16_view(h, 2) : h->w0));
          } else {
            if (off) TRY(rtm::stage_ready(h, slot));  // its staging slot's previous copy is done
            TRY(rtm::snap_prepare(h, slot));
            pending = rtm::io_store(h, slot), pending_slot = slot;
          }
          h->stored[slot] = 1;
        } else if (h->stored[slot]) {
          if (h->snap_fmt == RTM_SNAP_AE) {
            TRY(rtm::ae_load(h, slot, h->ae_scratch));
            if (h->dbl)
              TRY(rtm::ic_double_explicit(h, slot, h->f16 ? rtm::f16_view(h, 2) : h->w0));
            else if (h->ic_opt == RTM_IC_INVERSION)
              TRY(rtm::ic_explicit(h, slot, h->f16 ? rtm::f16_view(h, 2) : h->w0));
            else
              pending = rtm::io_image_ae(h, slot);
          } else {
            if (off) {
              // this slot in its staging slot before the next kernel reads it, then
              // the next slots (consumed in decreasing order) fetched ahead
              if (h->stage_slot[slot % h->nstage] != slot) TRY(rtm::offload_h2d(h, slot));
              TRY(rtm::stage_ready(h, slot));
              for (int a = 1; a < h->nstage && slot - a >= 0; a++) {
                const int sn = slot - a;
                if (h->stored[sn] && h->stage_slot[sn % h->nstage] != sn) TRY(rtm::offload_h2d(h, sn));
              }
            }
            if (h->dbl)  // now, on this step's field (the pending term's)
              TRY(rtm::ic_double_explicit(h, slot, h->f16 ? rtm::f16_view(h, 2) : h->w0));
            else if (h->ic_opt == RTM_IC_INVERSION)
              TRY(rtm::ic_explicit(h, slot, h->f16 ? rtm::f16_view(h, 2) : h->w0));
            else
              pending = rtm::io_image(h, slot);
          }
        }
      }
    }
    rtm::do_swap(h);
    return (int)RTM_OK;
  });
  if (rc != RTM_OK) return rc;
  if (pending.store || pending.ic) {  // the last step's snapshot / image term
    rtm::KScope k(h, RTM_K_IO);
    rtm::launch_fused_io(pending, h->f16 ? rtm::f16_view(h, 1) : h->w1, h->d.nx, h->d.ny, h->d.nz, h->st);
    TRY(rtm::check_launch(h, "fused_io(last)"));
    if (off && pending.store) TRY(rtm::offload_d2h(h, pending_slot));
    TRY(rtm::stage_join(h));
    CK(cudaStreamSynchronize(h->st));
  }
  return RTM_OK;
}

int rtm_get(rtm_handle *h, int field, float *dst) {
  if (!h || !dst) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  const float *src = field == RTM_FIELD_W0 ? (h->f16 ? rtm::f16_view(h, 0) : h->w0)
                     : field == RTM_FIELD_W1 ? (h->f16 ? rtm::f16_view(h, 1) : h->w1)
                     : field == RTM_FIELD_VEL ? h->vel
                     : field == RTM_FIELD_IMAGE ? h->image
                     : field == RTM_FIELD_INVQ ? h->invq
                     : field == RTM_FIELD_ILLUM ? h->illum : nullptr;
  if (!src) return RTM_ERR_ARG;
  CK(cudaMemcpyAsync(dst, src, 4 * (size_t)h->n, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_check_finite(rtm_handle *h, int field, int *nonfinite) {
  if (!h || !nonfinite) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  const float *src = field == RTM_FIELD_W0   ? (h->f16 ? rtm::f16_view(h, 0) : h->w0)
                     : field == RTM_FIELD_W1 ? (h->f16 ? rtm::f16_view(h, 1) : h->w1)
                     : field == RTM_FIELD_IMAGE ? h->image
                                                : nullptr;
  if (!src) return RTM_ERR_ARG;
  if (!h->nfflag) TRY(h->alloc(h->nfflag, 1));
  int f = 0;
  CK(cudaMemsetAsync(h->nfflag, 0, sizeof(int), h->st));
  rtm::launch_nonfinite_scan(src, h->n, h->nfflag, h->st);
  TRY(rtm::check_launch(h, "nonfinite_scan"));
  CK(cudaMemcpyAsync(&f, h->nfflag, sizeof f, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  *nonfinite = f != 0;
  return RTM_OK;
}

int rtm_selftest_bounded_wait(rtm_handle *h) {
  if (!h) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  rtm::launch_selftest_wait(h->dflag, h->st);
  TRY(rtm::check_launch(h, "selftest_wait"));
  CK(cudaStreamSynchronize(h->st));
  return rtm::check_flag(h);
}

int rtm_put(rtm_handle *h, int field, const float *src) {
  if (!h || !src || (field != RTM_FIELD_W0 && field != RTM_FIELD_W1)) return RTM_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->f16) {  // through the px scratch: slab max, scale, FP16 codes
    CK(cudaMemcpyAsync(h->px, src, 4 * (size_t)h->n, cudaMemcpyHostToDevice, h->st));
    const bool w0 = field == RTM_FIELD_W0;
    rtm::launch_f32_to_f16(h->px, w0 ? h->h0 : h->h1, w0 ? h->s0 : h->s1, w0 ? h->m0 : h->m1, h->d.ny, h->nxz,
                           h->f16_floor, h->st);
    TRY(rtm::check_launch(h, "f32_to_f16"));
  } else {
    CK(cudaMemcpyAsync(field == RTM_FIELD_W0 ? h->w0 : h->w1, src, 4 * (size_t)h->n, cudaMemcpyHostToDevice, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_c16_compress(const float *in, unsigned short *out, int nx, int ny, int nz) {
  // the encode kernel runs one grid row per y slab (gridDim.y <= 65535)
  if (!in || !out || nx < 1 || ny < 1 || nz < 1 || ny > 65535) return RTM_ERR_ARG;
  const size_t n = (size_t)nx * ny * nz, nc = ((size_t)nx * nz + 2) * ny;
  float *din = nullptr, *slab = nullptr;
  uint16_t *dout = nullptr;
  cudaStream_t st = 0;
  int rc = RTM_OK;
  if (cudaMalloc(&din, n * 4) || cudaMalloc(&dout, nc * 2) || cudaMalloc(&slab, ny * 4)) rc = RTM_ERR_NOMEM;
  if (rc == RTM_OK && cudaMemcpy(din, in, n * 4, cudaMemcpyHostToDevice)) rc = RTM_ERR_CUDA;
  if (rc == RTM_OK) {
    rtm::launch_c16_compress(din, dout, slab, nx, ny, nz, st);
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(out, dout, nc * 2, cudaMemcpyDeviceToHost)) rc = RTM_ERR_CUDA;
  }
  cudaFree(din), cudaFree(dout), cudaFree(slab);
  cudaGetLastError();
  return rc;
}

int rtm_c16_uncompress(const unsigned short *in, float *out, int nx, int ny, int nz) {
  // the decode kernel runs one grid layer per y slab (gridDim.z <= 65535)
  if (!in || !out || nx < 1 || ny < 1 || nz < 1 || ny > 65535) return RTM_ERR_ARG;
  const size_t n = (size_t)nx * ny * nz, nc = ((size_t)nx * nz + 2) * ny;
  float *dout = nullptr, *slab = nullptr, *ex = nullptr, *ey = nullptr, *ez = nullptr;
  uint16_t *din = nullptr;
  int rc = RTM_OK;
  if (cudaMalloc(&din, nc * 2) || cudaMalloc(&dout, n * 4) || cudaMalloc(&slab, ny * 4) || cudaMalloc(&ex, nx * 4) ||
      cudaMalloc(&ey, ny * 4) || cudaMalloc(&ez, nz * 4))
    rc = RTM_ERR_NOMEM;
  std::vector<float> tx, ty, tz;
  rtm::edge_taper(nx, 20, tx), rtm::edge_taper(ny, 20, ty), rtm::edge_taper(nz, 10, tz);
  if (rc == RTM_OK && (cudaMemcpy(din, in, nc * 2, cudaMemcpyHostToDevice) ||
                       cudaMemcpy(ex, tx.data(), nx * 4, cudaMemcpyHostToDevice) ||
                       cudaMemcpy(ey, ty.data(), ny * 4, cudaMemcpyHostToDevice) ||
                       cudaMemcpy(ez, tz.data(), nz * 4, cudaMemcpyHostToDevice)))
    rc = RTM_ERR_CUDA;
  if (rc == RTM_OK) {
    rtm::launch_c16_uncompress(din, dout, slab, ex, ey, ez, nx, ny, nz, 0);
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(out, dout, n * 4, cudaMemcpyDeviceToHost)) rc = RTM_ERR_CUDA;
  }
  cudaFree(din), cudaFree(dout), cudaFree(slab), cudaFree(ex), cudaFree(ey), cudaFree(ez);
  cudaGetLastError();
  return rc;
}

int rtm_batch_create(rtm_handle *const *shots, int nshots, rtm_batch **out) {
  if (!shots || nshots < 1 || !out) return RTM_ERR_ARG;
  *out = nullptr;
  rtm_batch *b = new rtm_batch();
  for (int k = 0; k < nshots; k++) {
    rtm::Engine *h = shots[k];
    // every shot ISO on the Laplacian kernel, or every shot FD8 VTI (or TTI) on
    // the two passes, leapfrog without Q or density, FP32 state, one device and
    // PML mode
    const bool iso = h && h->lap_iso();
    const bool aniso = h && h->c.engine == RTM_ENGINE_FD8 && h->c.model_type >= RTM_VTI && !h->c.use_rho && !h->f16;
    if (!h || !h->model_set || !(iso || aniso) || h->c.use_q || h->c.model_type != shots[0]->c.model_type ||
        h->device != shots[0]->device || h->c.pml3d != shots[0]->c.pml3d) {
      delete b;
      return !h || !h->model_set ? RTM_ERR_STATE : RTM_ERR_UNSUPPORTED;
    }
    b->shots.push_back(h);
  }
  b->device = shots[0]->device, b->pml3d = shots[0]->c.pml3d, b->model = shots[0]->c.model_type;
  cudaSetDevice(b->device);
  if (cudaStreamCreate(&b->st) || cudaEventCreate(&b->ev0) ||  // blocking: ordered after the set-up uploads
      cudaEventCreate(&b->ev1)) {
    cudaGetLastError();
    rtm_batch_destroy(b);
    return RTM_ERR_CUDA;
  }
  *out = b;
  return RTM_OK;
}

int rtm_batch_destroy(rtm_batch *b) {
  if (!b) return RTM_ERR_ARG;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  cudaFree(b->d_shots), cudaFree(b->d_ashots), cudaFree(b->d_start);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return RTM_OK;
}

int rtm_batch_modelling(rtm_batch *b, const int *nts, int it_shift, int ntratio) {
  if (!b || !nts || ntratio < 1) return RTM_ERR_ARG;
  cudaSetDevice(b->device);
  const int n = (int)b->shots.size();
  for (int k = 0; k < n; k++)
    if (nts[k] < 0) return RTM_ERR_ARG;
  // every handle's own stream must be idle before the batch stream touches its buffers
  for (rtm::Engine *h : b->shots) CK(cudaStreamSynchronize(h->st));
  std::vector<int> order(n);
  for (int k = 0; k < n; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return nts[x] > nts[y]; });
  std::vector<int> sorted(n);
  for (int k = 0; k < n; k++) sorted[k] = nts[order[k]];
  TRY(rtm::batch_run(b, order, sorted, sorted.empty() ? 0 : sorted[0], it_shift, ntratio));
  // each shot swapped its wavefields once per step
  for (int k = 0; k < n; k++)
    if (nts[k] & 1) {
      std::swap(b->shots[k]->w0, b->shots[k]->w1);
      b->shots[k]->iq0 = 1 - b->shots[k]->iq0;
    }
  return RTM_OK;
}

int rtm_batch_last_ms(rtm_batch *b, float *ms) {
  if (!b || !ms) return RTM_ERR_ARG;
  *ms = b->last_ms;
  return RTM_OK;
}

int rtm_batch_autotune(rtm_batch *b, int steps, int *choice) {
  if (!b || steps < 1) return RTM_ERR_ARG;
  cudaSetDevice(b->device);
  const int n = (int)b->shots.size();
  for (rtm::Engine *h : b->shots) CK(cudaStreamSynchronize(h->st));
  std::vector<int> order(n), sorted(n, steps);
  for (int k = 0; k < n; k++) order[k] = k;
  float best = 1e30f;
  int bi = 0;
  for (int c = 0; c < rtm::kBatchNShapes; c++) {
    if (b->model != RTM_ISO && rtm::kBatchShapes[c][0] != rtm::kAnisoBatchTX) continue;
    b->tx = rtm::kBatchShapes[c][0], b->yseg = rtm::kBatchShapes[c][1];
    TRY(rtm::batch_run(b, order, sorted, 1, 0, 0));  // warm-up
    TRY(rtm::batch_run(b, order, sorted, steps, 0, 0));
    if (b->last_ms < best) best = b->last_ms, bi = c;
  }
  b->tx = rtm::kBatchShapes[bi][0], b->yseg = rtm::kBatchShapes[bi][1];
  for (rtm::Engine *h : b->shots) {
    TRY(rtm::zero_state(h));
    CK(cudaStreamSynchronize(h->st));
  }
  if (choice) *choice = bi;
  return RTM_OK;
}

int rtm_autotune(rtm_handle *h, int steps, int *choice) {
  TRY(rtm::ready(h));
  if (steps < 1) return RTM_ERR_ARG;
  // candidate launch shapes of this handle's step kernels
  struct Cand {
    int iso4, v4, yseg;  // iso4 kind, its tile width (1) or shape (2), its y segment
    int tma_shape, tx, cfd_xy;
    int an4 = 0;  // FD8 VTI / TTI 4-cell kernels (y segment in yseg)
  };
  std::vector<Cand> cands;
  const bool iso = h->lap_iso();
  const bool v4_ok = iso && h->d.nz % 4 == 0 &&
                     (h->c.kernel_variant == 0 || h->c.kernel_variant == 3 || h->c.kernel_variant == 4);
  const int iso4_0 = h->iso4, v4_tx0 = h->v4_tx, v4_shape0 = h->v4_shape;
  // kind 1: tile width v, kind 2: TMA shape v; the modelled y segment and 32 planes
  auto add_iso4 = [&](int kind, int v) {
    h->iso4 = kind;
    if (kind == 1) h->v4_tx = v;
    else h->v4_shape = v;
    const int ym = rtm::yseg_iso4(h);
    cands.push_back({kind, v, ym, h->tma_shape, h->tx, h->cfd_xy});
    for (int y : {32, 64})
      if (ym != y && h->d.ny > y) cands.push_back({kind, v, y, h->tma_shape, h->tx, h->cfd_xy});
  };
  if (v4_ok) {
    for (int tx : {8, 16, 32}) add_iso4(1, tx);
    if (iso4_0 == 2)
      for (int k = 0; k < rtm::kIso4TmaNShapes; k++) add_iso4(2, k);
    h->iso4 = iso4_0, h->v4_tx = v4_tx0, h->v4_shape = v4_shape0;
  }
  if (iso && h->use_tma)
    for (int k = 0; k < rtm::kIsoTmaNShapes; k++) cands.push_back({0, 0, 0, k, h->tx, h->cfd_xy});
  else if (h->c.engine == RTM_ENGINE_FD8 && !v4_ok)
    for (int tx : {4, 8, 16}) cands.push_back({0, 0, 0, h->tma_shape, tx, h->cfd_xy});
  const int an4_0 = h->aniso4;
  if (an4_0) {
    const int ym = rtm::yseg_an4(h);
    cands.push_back({0, 0, ym, h->tma_shape, h->tx, h->cfd_xy, 1});
    for (int y : {32, 64})
      if (ym != y && h->d.ny > y) cands.push_back({0, 0, y, h->tma_shape, h->tx, h->cfd_xy, 1});
  }
  else if ((h->c.engine == RTM_ENGINE_CFD || h->c.engine == RTM_ENGINE_CFDB) && h->c.kernel_variant == 0) {
    if (h->cfd_seg_ok) {
      if (h->cfd_tma) cands.push_back({0, 0, 0, h->tma_shape, h->tx, 3});
      cands.push_back({0, 0, 0, h->tma_shape, h->tx, 4});
    }
    cands.push_back({0, 0, 0, h->tma_shape, h->tx, 0});
    if (h->cfd_tma) cands.push_back({0, 0, 0, h->tma_shape, h->tx, 1});
  }
  if (cands.empty()) {
    if (choice) *choice = 0;
    return RTM_OK;
  }
  const int yseg0 = h->yseg;
  auto apply = [&](const Cand &c) {
    if (an4_0) {
      h->aniso4 = c.an4;
      if (c.an4) {
        h->an4_yseg = c.yseg;
        TRY(rtm::an4_tiles(h));
      }
    }
    h->iso4 = c.iso4;
    if (c.iso4 == 1) h->v4_tx = c.v4;
    if (c.iso4 == 2) h->v4_shape = c.v4;
    if (c.iso4) h->v4_yseg = c.yseg;
    h->tma_shape = c.tma_shape, h->tx = c.tx, h->cfd_xy = c.cfd_xy;
    h->yseg = iso && h->use_tma ? yseg0 : rtm::yseg_for(h, h->tx);
    if (h->c.engine == RTM_ENGINE_FD8 && !h->lap_iso()) TRY(rtm::fd8_tiles(h));
    return h->iso4 == 2 ? rtm::iso4_tiles(h) : (int)RTM_OK;
  };
  float best = 1e30f;
  int bi = 0;
  h->tune_desc.clear(), h->tune_ms.clear();
  for (size_t c = 0; c < cands.size(); c++) {
    TRY(apply(cands[c]));
    TRY(rtm::step_kernel(h, 1, rtm::io_none()));  // warm-up (tensor maps, first launch)
    CK(cudaEventRecord(h->ev0, h->st));
    for (int s = 0; s < steps; s++) TRY(rtm::step_kernel(h, 1, rtm::io_none()));
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (ms < best) best = ms, bi = (int)c;
    const Cand &k = cands[c];
    const int fam = k.an4 ? 4 : k.iso4 ? k.iso4 : (iso && h->use_tma ? 3 : 0);
    h->tune_desc.push_back({fam, k.an4 ? rtm::kAniso4TX : k.iso4 ? k.v4 : fam == 3 ? k.tma_shape : k.tx,
                            k.iso4 || k.an4 ? k.yseg : 0, k.cfd_xy});
    h->tune_ms.push_back(ms);
  }
  TRY(apply(cands[bi]));
  if (choice) *choice = bi;
  TRY(rtm::check_flag(h));
  TRY(rtm::zero_state(h));
  CK(cudaStreamSynchronize(h->st));
  return RTM_OK;
}

int rtm_autotune_result(rtm_handle *h, int idx, int desc[4], float *ms) {
  if (!h || !desc || !ms || idx < 0 || idx >= (int)h->tune_ms.size()) return RTM_ERR_ARG;
  for (int k = 0; k < 4; k++) desc[k] = h->tune_desc[idx][k];
  *ms = h->tune_ms[idx];
  return RTM_OK;
}

int rtm_profile(rtm_handle *h, int on) {
  if (!h) return RTM_ERR_ARG;
  h->prof_on = on ? 1 : 0;
  for (int k = 0; k < RTM_NKINDS; k++) h->prof_ms[k] = 0.0, h->prof_cnt[k] = 0;
  return RTM_OK;
}

int rtm_profile_read(rtm_handle *h, double *ms, long long *count) {
  if (!h || !ms || !count) return RTM_ERR_ARG;
  for (int k = 0; k < RTM_NKINDS; k++) ms[k] = h->prof_ms[k], count[k] = h->prof_cnt[k];
  return RTM_OK;
}

int rtm_last_loop_launches(rtm_handle *h, long long *n) {
  if (!h || !n) return RTM_ERR_ARG;
  *n = h->launches;
  return RTM_OK;
}

int rtm_last_loop_ms(rtm_handle *h, float *ms) {
  if (!h || !ms) return RTM_ERR_ARG;
  *ms = h->last_ms;
  return RTM_OK;
}

}  // extern "C"
