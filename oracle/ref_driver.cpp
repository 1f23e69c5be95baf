// ref_driver.cpp - harness around the reference's OWN compiled CPU kernels.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  Linked
// into oracle/_ref/libbgprtm_ref.so together with bgprtm's KernelCPU.cpp,
// FdEngine.cpp (lines 1-517), FdEngine_fd.cpp, FdEngine_cfd.cpp, Cfd_plan.cpp,
// PML.cpp, WaveFieldCompress.cpp and TimeRecorder.cpp, compiled from the
// reference tree by oracle/Makefile.  The spatial operator, the PML, the CFD
// plan and the snapshot codec are the reference's code; the time-loop glue
// around them (Propagator::Vel2 / update2nd, Receiver::apply_src) does not
// compile in the reference tree and is restated here from
// bgprtm/Propagator.cpp:711-742, 1767-1788 and bgprtm/Receiver.cpp:477-507.
#include <omp.h>
#include <xmmintrin.h>

#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "Cfd_plan.h"
#include "FdEngine.h"
#include "GetPar.h"
#include "KernelCPU.h"
#include "Util.h"
#include "volumefilter.h"
#include "PML.h"
#include "WaveFieldCompress.h"

namespace {
float *vol_alloc(size_t n) {  // bgprtm/Wavefield.cpp:183-192
  float *p = (float *)_mm_malloc(n * sizeof(float) + 128, 16);
  memset(p, 0, n * sizeof(float) + 128);
  return p;
}

struct RefHandle {
  int nx, ny, nz, model, engine, nthreads;
  float dt;
  size_t n;
  KernelCPU *k = nullptr;
  float *w0, *w1, *wr, *vel, *eps = nullptr, *del = nullptr, *pjx = nullptr, *pjy = nullptr, *rho = nullptr;
  // injection traces (restated Receiver::apply_src)
  int ntr = 0, lx = 0, ly = 0, lz = 0, nt = 0;
  std::vector<int> off, len;
  std::vector<float> kx, ky, kz, traces;
  float scaler = 1;
  // receivers (restated ExtractReceiverData::extract / Receiver::extract_value)
  int nrc = 0, rlx = 0, rly = 0, rlz = 0, nt_out = 0;
  std::vector<int> roff, rlen;
  std::vector<float> rkx, rky, rkz, out;
};

void set_globals(int engine, int model, float pml_eps, int pml3d, float scaler, int top_pml, int use_rho) {
  shim_store().kv.clear();
  global_pars["Engine"] = engine == 1 ? "CFD" : engine == 2 ? "FFTWR2C" : engine == 3 ? "FFTWR2R" : "FD";
  global_pars["fd_use_taylor"] = 1;
  global_pars["pml_eps"] = pml_eps;
  global_pars["pml3d"] = pml3d;
  global_pars["pml3d_scaler"] = scaler;
  global_pars["top_pml_flag"] = top_pml;
  global_pars["wf_compress"] = 1;
  // FdEngine::determineModelType decides dimPML (bgprtm/FdEngine.cpp:49-52,
  // 216-264).  For VTI with the FD engine isDerive2nd() is true, which
  // allocates one PML component while the first-derivative path indexes three
  // (a null dereference in the reference); force_tti=1 selects the allocation
  // the VTI path needs.
  if (model == 3) global_pars["global"]["pjx"] = 1;
  if (model == 2) global_pars["global"]["epsilon"] = 1, global_pars["force_tti"] = 1;
  // a density model sends ISO through KernelCPU::TTI (bgprtm/KernelCPU.cpp:128),
  // which needs the three-component PML allocation as above
  if (use_rho) global_pars["global"]["rho"] = 1, global_pars["force_tti"] = 1;
}
}  // namespace

extern "C" {

void *ref_create(int nx, int ny, int nz, float dx, float dy, float dz, float dt, int engine, int model,
                 const int *nbnd, float vmax, float pml_eps, int pml3d, float pml3d_scaler, int top_pml,
                 int nthreads, int use_rho) {
  if (engine < 0 || engine > 3) return nullptr;  // KernelCPU engines only (FD, CFD, FFTWR2C, FFTWR2R)
  set_globals(engine, model, pml_eps, pml3d, pml3d_scaler, top_pml, use_rho);
  RefHandle *h = new RefHandle();
  h->nx = nx, h->ny = ny, h->nz = nz, h->model = model, h->engine = engine, h->dt = dt;
  h->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
  h->n = (size_t)nx * ny * nz;
  h->w0 = vol_alloc(h->n), h->w1 = vol_alloc(h->n), h->wr = vol_alloc(h->n), h->vel = vol_alloc(h->n);
  h->k = new KernelCPU(nx, ny, nz, dx, dy, dz, engine == 1   ? FD::CFD
                       : engine == 2 ? FD::FFTWR2C
                       : engine == 3 ? FD::FFTWR2R
                                     : FD::FD,
                       h->nthreads);
  h->k->setJacob(nullptr, nullptr, nullptr, nullptr);
  h->k->setBoundary(nbnd[0], nbnd[1], nbnd[2], nbnd[3], nbnd[4], nbnd[5], dt, vmax);
  return h;
}

void ref_destroy(void *p) {
  RefHandle *h = (RefHandle *)p;
  delete h->k;
  for (float *a : {h->w0, h->w1, h->wr, h->vel, h->eps, h->del, h->pjx, h->pjy, h->rho})
    if (a) _mm_free(a);
  delete h;
}

// Propagator::Vel2, no-Q branch (bgprtm/Propagator.cpp:715-725); rho (may be
// null) goes to KernelCPU::setModel as Propagator passes volModel[RHO]
// (bgprtm/Propagator.cpp:299)
void ref_set_model(void *p, const float *v, const float *rho, const float *eps, const float *del, const float *pjx,
                   const float *pjy) {
  RefHandle *h = (RefHandle *)p;
  float dt2 = h->dt * h->dt;
  for (size_t i = 0; i < h->n; i++) h->vel[i] = (v[i] * v[i]) * dt2;
  auto cp = [&](float *&dst, const float *src) {
    if (!src) return;
    if (!dst) dst = vol_alloc(h->n);
    memcpy(dst, src, h->n * 4);
  };
  cp(h->eps, eps), cp(h->del, del), cp(h->pjx, pjx), cp(h->pjy, pjy), cp(h->rho, rho);
  h->k->setModel(h->vel, h->rho, h->del, h->eps, h->pjx, h->pjy);
}

void ref_reset(void *p) {
  RefHandle *h = (RefHandle *)p;
  memset(h->w0, 0, h->n * 4), memset(h->w1, 0, h->n * 4), memset(h->wr, 0, h->n * 4);
  h->k->cleanPMLMemory();
}

// Propagator::kernel, KernelCPU branch (bgprtm/Propagator.cpp:994-1001)
void ref_kernel(void *p) {
  RefHandle *h = (RefHandle *)p;
  if (h->model == 3) h->k->TTI(h->w1, h->w0, h->wr);
  else if (h->model == 2) h->k->VTI(h->w1, h->w0, h->wr);
  else h->k->ISO(h->w1, h->w0, h->wr, 0, 0, 0);
}

// Propagator::update2nd, no-Q branch (bgprtm/Propagator.cpp:1771-1788)
void ref_update2nd(void *p) {
  RefHandle *h = (RefHandle *)p;
  float *w0 = h->w0, *w1 = h->w1;
  size_t n = h->n;
#pragma omp parallel for num_threads(h->nthreads) schedule(static)
  for (long i = 0; i < (long)n; i += 4) {
    __m128 a = _mm_load_ps(w0 + i), b = _mm_load_ps(w1 + i);
    _mm_store_ps(w0 + i, _mm_sub_ps(_mm_add_ps(b, b), a));
  }
}

void ref_swap(void *p) {
  RefHandle *h = (RefHandle *)p;
  std::swap(h->w0, h->w1);
}

void ref_put(void *p, int field, const float *src) {
  RefHandle *h = (RefHandle *)p;
  memcpy(field == 0 ? h->w0 : h->w1, src, h->n * 4);
}
void ref_get(void *p, int field, float *dst) {
  RefHandle *h = (RefHandle *)p;
  const float *s = field == 0 ? h->w0 : field == 1 ? h->w1 : h->vel;
  memcpy(dst, s, h->n * 4);
}

void ref_set_injection(void *p, int ntr, int lx, int ly, int lz, const int *off, const int *len, const float *kx,
                       const float *ky, const float *kz, const float *tr, int nt, float scaler) {
  RefHandle *h = (RefHandle *)p;
  h->ntr = ntr, h->lx = lx, h->ly = ly, h->lz = lz, h->nt = nt, h->scaler = scaler;
  h->off.assign(off, off + 3 * ntr), h->len.assign(len, len + 3 * ntr);
  h->kx.assign(kx, kx + (size_t)ntr * lx), h->ky.assign(ky, ky + (size_t)ntr * ly);
  h->kz.assign(kz, kz + (size_t)ntr * lz), h->traces.assign(tr, tr + (size_t)ntr * nt);
}

// Receiver::apply_src for every trace (bgprtm/Receiver.cpp:477-507)
void ref_inject(void *p, int it) {
  RefHandle *h = (RefHandle *)p;
  if (it < 0 || it >= h->nt) return;
  for (int r = 0; r < h->ntr; r++) {
    float val = h->traces[(size_t)r * h->nt + it] * h->scaler;
    const int *o = &h->off[3 * r], *l = &h->len[3 * r];
    for (int iy = 0; iy < l[1]; iy++) {
      float cy = val * h->ky[(size_t)r * h->ly + iy];
      for (int ix = 0; ix < l[0]; ix++) {
        float cx = cy * h->kx[(size_t)r * h->lx + ix];
        size_t off = ((size_t)(iy + o[1]) * h->nx + ix + o[0]) * h->nz + o[2];
        for (int iz = 0; iz < l[2]; iz++) h->w0[off + iz] += cx * h->kz[(size_t)r * h->lz + iz] * h->vel[off + iz];
      }
    }
  }
}

void ref_set_extraction(void *p, int ntr, int lx, int ly, int lz, const int *off, const int *len, const float *kx,
                        const float *ky, const float *kz, int nt_out) {
  RefHandle *h = (RefHandle *)p;
  h->nrc = ntr, h->rlx = lx, h->rly = ly, h->rlz = lz, h->nt_out = nt_out;
  h->roff.assign(off, off + 3 * ntr), h->rlen.assign(len, len + 3 * ntr);
  h->rkx.assign(kx, kx + (size_t)ntr * lx), h->rky.assign(ky, ky + (size_t)ntr * ly);
  h->rkz.assign(kz, kz + (size_t)ntr * lz);
  h->out.assign((size_t)ntr * nt_out, 0.f);
}

// Receiver::extract_value for every receiver (bgprtm/Receiver.cpp:394-426),
// sample jt
void ref_extract(void *p, int jt) {
  RefHandle *h = (RefHandle *)p;
  if (jt < 0 || jt >= h->nt_out) return;
#pragma omp parallel for num_threads(h->nthreads) schedule(static)
  for (int r = 0; r < h->nrc; r++) {
    float val = 0.f;
    const int *o = &h->roff[3 * r], *l = &h->rlen[3 * r];
    for (int iy = 0; iy < l[1]; iy++) {
      float cy = h->rky[(size_t)r * h->rly + iy];
      for (int ix = 0; ix < l[0]; ix++) {
        float cx = cy * h->rkx[(size_t)r * h->rlx + ix];
        size_t off = ((size_t)(iy + o[1]) * h->nx + ix + o[0]) * h->nz + o[2];
        for (int iz = 0; iz < l[2]; iz++) val += cx * h->rkz[(size_t)r * h->rlz + iz] * h->w0[off + iz];
      }
    }
    h->out[(size_t)r * h->nt_out + jt] = val;
  }
}
void ref_get_traces(void *p, float *dst) {
  RefHandle *h = (RefHandle *)p;
  std::copy(h->out.begin(), h->out.end(), dst);
}

// Propagator::modelling's loop body (bgprtm/Propagator.cpp:1099-1153): kernel,
// update2nd, inject(it + it_shift), extract(it / ntratio), swap
void ref_modelling(void *p, int nts, int it_shift, int ntratio) {
  for (int it = 0; it < nts; it++) {
    ref_kernel(p);
    ref_update2nd(p);
    ref_inject(p, it + it_shift);
    if (it % ntratio == 0) ref_extract(p, it / ntratio);
    ref_swap(p);
  }
}

// K steps of the forward loop body (kernel, update2nd, inject, swap), wall
// seconds.  The reference's CPU time-step cost, used as the CPU baseline.
double ref_run(void *p, int it0, int nsteps) {
  auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < nsteps; s++) {
    ref_kernel(p);
    ref_update2nd(p);
    ref_inject(p, it0 + s - 1);
    ref_swap(p);
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The reference's snapshot codec (bgprtm/WaveFieldCompress.cpp:135-207).
void ref_c16_compress(const float *in, unsigned short *out, int nx, int ny, int nz) {
  global_pars["wf_compress"] = 1;
  WaveFieldCompress c(1);
  c.compress(const_cast<float *>(in), out, nx, ny, nz);
}
void ref_c16_uncompress(const unsigned short *in, float *out, int nx, int ny, int nz) {
  global_pars["wf_compress"] = 1;
  WaveFieldCompress c(1);
  c.uncompress(const_cast<unsigned short *>(in), out, nx, ny, nz);
}

// The reference's CFD plan (bgprtm/Cfd_plan.cpp): s = 0 -> isgn 1, s = 1 -> isgn 2.
void ref_cfd_plan(int n, float d, int s, float *bm, float *bl, float *am) {
  CfdPlan c(n, d);
  memcpy(bm, s ? c.bm2 : c.bm1, sizeof(float) * 5 * n);
  memcpy(bl, s ? c.bl2 : c.bl1, sizeof(float) * 4 * n);
  memcpy(am, s ? c.am2 : c.am1, sizeof(float) * 60);
}

// The reference's PML damping profile (bgprtm/PML.cpp:87-124).
void ref_pml_coef(int n, int npml, float d, float dt, float vmax, float pml_eps, float *coef) {
  global_pars["pml_eps"] = pml_eps;
  PML pml(n, npml, 1, d, dt, vmax, false);
  memcpy(coef, pml.coef.data(), sizeof(float) * npml);
}

// Util::CompactOrmsbySpreadCoeff with a kernel-length cap; returns the first index
int ref_spread_coeffs(int n, float x, float k1, float k2, int *nlimit, int dipole, float *coeff) {
  return Util::CompactOrmsbySpreadCoeff(n, coeff, x, k1, k2, nlimit, dipole != 0, false);
}

// volumefilter.cpp's running box averages (illumination smoothing), in place
void ref_avg_volume3d(float *a, int nx, int ny, int nz, int sx, int sy, int sz) { avgVolume3D(a, nx, ny, nz, sx, sy, sz); }
void ref_avg_volume2d(float *a, int nx, int nz, int sx, int sz) { avgVolume2D(a, nx, nz, sx, sz); }
}
