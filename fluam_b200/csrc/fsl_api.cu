// fsl_api.cu -- the C ABI of libfluamsl (declared in include/fluamsl.h):
// device state of one Stokes-limit instance, the per-step launch sequence
// (captured in a CUDA graph), and the component entry points.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/fluamsl.h"
#include "fsl_internal.cuh"

namespace {
thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define FSL_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return set_error(e_ == cudaErrorMemoryAllocation ? FSL_E_NOMEM : FSL_E_CUDA,        \
                       "%s failed: %s", #call, cudaGetErrorString(e_));                  \
  } while (0)

}  // namespace

int fsl::set_last_error(int code, const char* msg) { return set_error(code, "%s", msg); }

namespace {

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMalloc((void**)p, sizeof(T) * n);
}
}  // namespace

struct fsl_handle {
  fsl::Params P;
  int device = 0;
  cudaStream_t stream = nullptr;
  fsl::FftPlan* fft = nullptr;
  // particles
  double *q = nullptr, *qp = nullptr, *F = nullptr;
  // cell list
  int *cell_of = nullptr, *cnt = nullptr, *start = nullptr, *fill = nullptr, *tmp = nullptr,
      *sorted = nullptr, *bsum = nullptr;
  // bonds
  int *bpp_cnt = nullptr, *bpp_off = nullptr, *bpp_idx = nullptr;
  double *bpp_k = nullptr, *bpp_r0 = nullptr;
  int *bfp_cnt = nullptr, *bfp_off = nullptr;
  double *bfp_k = nullptr, *bfp_r0 = nullptr, *bfp_xyz = nullptr;
  float* ljtab = nullptr;
  // fields
  float* noise = nullptr;
  unsigned long long* grid = nullptr;
  float2* spec = nullptr;
  float* v = nullptr;
  // scratch for the component entry points (allocated on first use)
  float* wext = nullptr;
  float* wbuf = nullptr;  // W of the current solve, [3][nc]
  double* u = nullptr;
  float* nbuf = nullptr;
  int64_t nbuf_n = 0;
  int* err = nullptr;
  uint64_t* t_dev = nullptr;
  uint64_t steps = 0;
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  fsl::Prof prof;
  std::map<std::string, std::pair<int64_t, double>> stage_acc;
  int launches_per_step = 0;
};

namespace {

void free_all(fsl_handle* h) {
  if (!h) return;
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  void* ptrs[] = {h->q,       h->qp,      h->F,       h->cell_of, h->cnt,     h->start,
                  h->fill,    h->tmp,     h->sorted,  h->bsum,    h->bpp_cnt, h->bpp_off,
                  h->bpp_idx, h->bpp_k,   h->bpp_r0,  h->bfp_cnt, h->bfp_off, h->bfp_k,
                  h->bfp_r0,  h->bfp_xyz, h->ljtab,   h->noise,   h->grid,    h->spec,
                  h->v,       h->wext,    h->u,       h->nbuf,    h->err,     h->t_dev,
                  h->wbuf};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < fsl::Prof::kMax; ++i)
    if (h->prof.ev[i]) cudaEventDestroy(h->prof.ev[i]);
  fsl::fft_plan_destroy(h->fft);
  if (h->stream) cudaStreamDestroy(h->stream);
}

// src/initForcesNonBonded.cu:21-53 (float accumulation, float sqrt, sigma =
// 2 dx, epsilon = kT, first and last entries zero).
void build_ljtable(const fsl::Params& P, double temperature, double cutoff, std::vector<float>& t) {
  const int size = fsl::kLjTableSize;
  t.assign(size, 0.0f);
  float sigma = (float)(2.0 * P.lx / (double)P.mx);
  float epsilon = (float)temperature;
  float cutoff2 = (float)(cutoff * cutoff);
  float dr = cutoff2 / (float)size;
  float r = 0.5f * dr;
  for (int i = 0; i < size; ++i) {
    double rr = (double)sqrtf(r);
    float fr = (float)(48. * epsilon * (std::pow(sigma / rr, 12) - 0.5 * std::pow(sigma / rr, 6)) / rr);
    t[i] = fr / sqrtf(r);
    r += dr;
  }
  t[size - 1] = 0.0f;
  t[0] = 0.0f;
}

void enqueue_cells_forces(fsl_handle* h, const double* pos) {
  const fsl::Params& P = h->P;
  fsl::Prof& pr = h->prof;
  pr.mark(h->stream, "cells");
  fsl::launch_cells(P, pos, h->cell_of, h->cnt, h->start, h->fill, h->tmp, h->sorted, h->bsum, h->err,
                    h->stream);
  pr.mark(h->stream, "forces");
  fsl::launch_forces(P, pos, h->cell_of, h->start, h->sorted, h->bpp_cnt, h->bpp_off, h->bpp_idx,
                     h->bpp_k, h->bpp_r0, h->bfp_cnt, h->bfp_off, h->bfp_k, h->bfp_r0, h->bfp_xyz,
                     h->ljtab, h->F, h->err, h->stream);
  if (P.np > 0) pr.count(7);
}

// One midpoint step (src/runSchemeStokesLimit.cu:163-275).
void enqueue_step(fsl_handle* h) {
  const fsl::Params& P = h->P;
  cudaStream_t s = h->stream;
  fsl::Prof& pr = h->prof;
  pr.used = 0;
  pr.launches = 0;
  const size_t gbytes = sizeof(unsigned long long) * 3 * (size_t)P.nc;
  const int pk = P.np > 0 ? 1 : 0;
  pr.mark(s, "noise");
  fsl::launch_noise(P, h->t_dev, h->noise, s);
  pr.count(1);
  // option 0: F^n, f = S(q^n) F^n; solve 1 with sqrt(2) stress 1.  The
  // spread field is all zeros here: it is cleared at creation and by every
  // W build that reads it.
  (void)gbytes;
  enqueue_cells_forces(h, h->q);
  pr.mark(s, "spread");
  fsl::launch_spread(P, 0, h->sorted, h->q, h->F, h->q, h->noise, h->grid, h->err, s);
  pr.count(pk);
  fsl::launch_solve(P, h->fft, h->grid, h->noise, 1, nullptr, h->wbuf, h->spec, h->v, s, &pr);
  // option 1: predictor, F^{n+1/2}, f = S F + RFD; solve 2 with sqrt(1/2)(stress 1 + 2)
  pr.mark(s, "interp_update");
  fsl::launch_interp_update(P, 1, h->q, h->q, h->F, h->noise, h->v, h->qp, h->err, s);
  pr.count(pk);
  enqueue_cells_forces(h, h->qp);
  pr.mark(s, "spread_rfd");
  fsl::launch_spread(P, 1, h->sorted, h->qp, h->F, h->q, h->noise, h->grid, h->err, s);
  pr.count(pk);
  fsl::launch_solve(P, h->fft, h->grid, h->noise, 2, nullptr, h->wbuf, h->spec, h->v, s, &pr);
  // option 2: corrector
  pr.mark(s, "interp_update");
  fsl::launch_interp_update(P, 2, h->qp, h->q, h->F, h->noise, h->v, h->q, h->err, s);
  pr.count(pk);
  pr.mark(s, "counter");
  fsl::launch_step_counter(h->t_dev, s);
  pr.count(1);
  pr.mark(s, nullptr);
  h->launches_per_step = pr.launches;
}

// Charge the event intervals of the last step to their stages.
int prof_collect(fsl_handle* h) {
  fsl::Prof& pr = h->prof;
  if (!pr.on || pr.used < 2) return FSL_OK;
  cudaError_t e = cudaEventSynchronize(pr.ev[pr.used - 1]);
  if (e != cudaSuccess) return set_error(FSL_E_CUDA, "profile sync: %s", cudaGetErrorString(e));
  for (int i = 0; i + 1 < pr.used; ++i) {
    if (!pr.name[i]) continue;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pr.ev[i], pr.ev[i + 1]);
    auto& a = h->stage_acc[pr.name[i]];
    a.first += 1;
    a.second += ms;
  }
  return FSL_OK;
}

void drop_graph(fsl_handle* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->gexec = nullptr;
  h->graph = nullptr;
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(FSL_E_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  return FSL_OK;
}

bool factor_ok(int n) {
  if (n < 3) return false;
  const int ps[5] = {2, 3, 5, 7, 11};
  for (int p : ps)
    while (n % p == 0) n /= p;
  return n == 1;
}

}  // namespace

extern "C" {

const char* fsl_last_error(void) { return g_err; }

void fsl_config_defaults(fsl_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->mx = c->my = c->mz = 32;
  c->lx = c->ly = c->lz = 32.0;
  c->kernel = 3;
  c->shearviscosity = 1.0;
  c->temperature = 0.0;
  c->dt = 0.0;
  c->cutoff = 0.0;  // src/loadDataMain.cu:192
  c->extra_mobility = 0.0;
  c->soft_epsilon = 1.0;
  c->seed = 0;
  c->pair = FSL_PAIR_TABLE_LJ;
  c->rfd = FSL_RFD_REFERENCE;
  c->nonbonded = 1;  // src/loadDataMain.cu:206
  c->device = -1;    // src/loadDataMain.cu:181
}

int fsl_create(const fsl_config* cfg, int64_t np, const double* q, fsl_handle** out) {
  if (!cfg || !out) return set_error(FSL_E_ARG, "null argument");
  *out = nullptr;
  const fsl_config& c = *cfg;
  if (c.mx < 3 || c.my < 3 || c.mz < 3)
    return set_error(FSL_E_ARG, "cells must be >= 3 in every direction");
  if (!factor_ok(c.mx) || !factor_ok(c.my) || !factor_ok(c.mz))
    return set_error(FSL_E_ARG, "cells %d %d %d: every extent must factor into 2,3,5,7,11", c.mx,
                     c.my, c.mz);
  if (c.mx > 1024 || c.my > 1024 || c.mz > 1024)
    return set_error(FSL_E_ARG, "cells per direction limited to 1024");
  if (!(c.lx > 0 && c.ly > 0 && c.lz > 0)) return set_error(FSL_E_ARG, "celldimension must be > 0");
  if (!(c.dt > 0)) return set_error(FSL_E_ARG, "dt must be > 0");
  if (!(c.shearviscosity > 0)) return set_error(FSL_E_ARG, "shearviscosity must be > 0");
  if (!(c.temperature >= 0)) return set_error(FSL_E_ARG, "temperature must be >= 0");
  if (c.kernel != 3 && c.kernel != 4) return set_error(FSL_E_ARG, "kernel must be 3 or 4");
  if (c.pair < 0 || c.pair > 2) return set_error(FSL_E_ARG, "unknown pair potential %d", c.pair);
  if (c.rfd < 0 || c.rfd > 1) return set_error(FSL_E_ARG, "unknown rfd mode %d", c.rfd);
  if (c.extra_mobility < 0) return set_error(FSL_E_ARG, "extraMobility must be >= 0");
  if (np < 0 || np > (int64_t)1 << 28) return set_error(FSL_E_ARG, "bad particle count");
  if (np > 0 && !q) return set_error(FSL_E_ARG, "null positions");
  bool pairs = c.nonbonded && c.pair != FSL_PAIR_NONE && np > 0;
  if (pairs && !(c.cutoff > 0)) return set_error(FSL_E_ARG, "cutoff must be > 0 with pair forces");
  int64_t nc64 = (int64_t)c.mx * c.my * c.mz;
  if (nc64 > ((int64_t)1 << 30)) return set_error(FSL_E_ARG, "grid too large");

  fsl_handle* h = new fsl_handle();
  fsl::Params& P = h->P;
  std::memset(&P, 0, sizeof(P));
  P.mx = c.mx;
  P.my = c.my;
  P.mz = c.mz;
  P.mxh = c.mx / 2 + 1;
  P.nc = (int)nc64;
  P.lx = c.lx;
  P.ly = c.ly;
  P.lz = c.lz;
  // src/createCellsStokesLimitGPU.cu:71-91
  P.dx = c.lx / double(c.mx);
  P.dy = c.ly / double(c.my);
  P.dz = c.lz / double(c.mz);
  P.invdx = double(c.mx) / c.lx;
  P.invdy = double(c.my) / c.ly;
  P.invdz = double(c.mz) / c.lz;
  P.invlx = 1. / c.lx;
  P.invly = 1. / c.ly;
  P.invlz = 1. / c.lz;
  P.dV = P.dx * P.dy * P.dz;
  // src/createBoundariesRK2GPU.cu:134-141
  if (c.cutoff > 0) {
    P.mnx = std::max(3, (int)(c.lx / c.cutoff));
    P.mny = std::max(3, (int)(c.ly / c.cutoff));
    P.mnz = std::max(3, (int)(c.lz / c.cutoff));
  } else {
    P.mnx = P.mny = P.mnz = 3;
  }
  if ((int64_t)P.mnx * P.mny * P.mnz > ((int64_t)1 << 28)) {
    delete h;
    return set_error(FSL_E_ARG, "cutoff too small for the box (neighbour grid too large)");
  }
  P.mN = P.mnx * P.mny * P.mnz;
  P.invdnx = double(P.mnx) / c.lx;
  P.invdny = double(P.mny) / c.ly;
  P.invdnz = double(P.mnz) / c.lz;
  P.np = (int)np;
  P.kernel = c.kernel;
  P.pair = c.pair;
  P.nonbonded = c.nonbonded ? 1 : 0;
  P.rfd = c.rfd;
  P.bonded = 0;
  P.has_extra = c.extra_mobility != 0.0;
  P.cutoff = c.cutoff;
  P.cutoff2 = c.cutoff * c.cutoff;
  P.invcut2 = c.cutoff > 0 ? 1. / (c.cutoff * c.cutoff) : 0.0;
  P.soft_eps = c.soft_epsilon;
  P.eta = c.shearviscosity;
  P.kT = c.temperature;
  P.dt = c.dt;
  P.extra_mob = c.extra_mobility;
  // src/createCellsStokesLimitGPU.cu:58-61
  P.fact1 = std::sqrt((4. * c.temperature * c.shearviscosity) / (P.dV * c.dt));
  P.fact4 = std::sqrt((2. * c.temperature * c.shearviscosity) / (P.dV * c.dt));
  P.fact2 = std::sqrt(c.temperature * c.extra_mobility * c.dt);
  P.seed = c.seed;
  P.noise_n = (uint64_t)12 * P.nc + (uint64_t)9 * P.np;

  auto fail = [&](int code) {
    free_all(h);
    delete h;
    return code;
  };
#define TRY(call)                                                                              \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return fail(set_error(e_ == cudaErrorMemoryAllocation ? FSL_E_NOMEM : FSL_E_CUDA,         \
                            "%s: %s", #call, cudaGetErrorString(e_)));                         \
  } while (0)
  if (c.device >= 0) TRY(cudaSetDevice(c.device));
  TRY(cudaGetDevice(&h->device));
  TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  const size_t n3p = 3 * (size_t)np, n3c = 3 * (size_t)P.nc;
  TRY(dalloc(&h->q, n3p));
  TRY(dalloc(&h->qp, n3p));
  TRY(dalloc(&h->F, n3p));
  TRY(dalloc(&h->cell_of, np));
  TRY(dalloc(&h->cnt, P.mN));
  TRY(dalloc(&h->start, (size_t)P.mN + 1));
  TRY(dalloc(&h->fill, P.mN));
  TRY(dalloc(&h->tmp, np));
  TRY(dalloc(&h->sorted, np));
  TRY(dalloc(&h->bsum, (P.mN + 4095) / 4096 + 1));
  TRY(dalloc(&h->bpp_cnt, np));
  TRY(dalloc(&h->bpp_off, np));
  TRY(dalloc(&h->bfp_cnt, np));
  TRY(dalloc(&h->bfp_off, np));
  TRY(dalloc(&h->ljtab, fsl::kLjTableSize));
  TRY(dalloc(&h->noise, (P.noise_n + 3) / 4 * 4));
  TRY(dalloc(&h->grid, n3c));
  TRY(dalloc(&h->spec, 3 * (size_t)P.my * P.mz * P.mxh));
  TRY(dalloc(&h->v, n3c));
  TRY(dalloc(&h->wbuf, n3c));
  TRY(cudaMemset(h->grid, 0, sizeof(unsigned long long) * n3c));
  TRY(dalloc(&h->err, 4));
  TRY(dalloc(&h->t_dev, 1));
  if ((int64_t)((P.mN + 4095) / 4096) > 4096) return fail(set_error(FSL_E_ARG, "neighbour grid too large"));
  TRY(cudaMemset(h->bpp_cnt, 0, sizeof(int) * std::max<int64_t>(np, 1)));
  TRY(cudaMemset(h->bfp_cnt, 0, sizeof(int) * std::max<int64_t>(np, 1)));
  TRY(cudaMemset(h->bpp_off, 0, sizeof(int) * std::max<int64_t>(np, 1)));
  TRY(cudaMemset(h->bfp_off, 0, sizeof(int) * std::max<int64_t>(np, 1)));
  TRY(cudaMemset(h->err, 0, sizeof(int) * 4));
  TRY(cudaMemset(h->t_dev, 0, sizeof(uint64_t)));
  TRY(cudaMemset(h->v, 0, sizeof(float) * n3c));
  TRY(cudaMemset(h->F, 0, sizeof(double) * std::max<size_t>(n3p, 1)));
  if (np > 0) {
    TRY(cudaMemcpy(h->q, q, sizeof(double) * n3p, cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(h->qp, q, sizeof(double) * n3p, cudaMemcpyHostToDevice));
  }
  std::vector<float> tab;
  build_ljtable(P, c.temperature, c.cutoff, tab);
  TRY(cudaMemcpy(h->ljtab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice));
  h->fft = fsl::fft_plan_create(P);
  if (!h->fft) return fail(set_error(FSL_E_ARG, "FFT plan creation failed (sizes or shared memory)"));
  TRY(cudaDeviceSynchronize());
#undef TRY
  *out = h;
  return FSL_OK;
}

void fsl_destroy(fsl_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
}

void* fsl_stream(fsl_handle* h) { return h ? (void*)h->stream : nullptr; }

int fsl_load_bonds(fsl_handle* h, int64_t nbonds, const int32_t* bi, const int32_t* bj,
                   const double* k, const double* r0, int64_t nfixed, const int32_t* fi,
                   const double* fk, const double* fr0, const double* fxyz) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  const int np = h->P.np;
  if (nbonds < 0 || nfixed < 0) return set_error(FSL_E_ARG, "negative bond count");
  for (int64_t b = 0; b < nbonds; ++b)
    if (bi[b] < 0 || bi[b] >= np || bj[b] < 0 || bj[b] >= np)
      return set_error(FSL_E_ARG, "bond %lld: particle index out of range", (long long)b);
  for (int64_t b = 0; b < nfixed; ++b)
    if (fi[b] < 0 || fi[b] >= np)
      return set_error(FSL_E_ARG, "tether %lld: particle index out of range", (long long)b);
  // CSR as src/initializeBondedForces.cpp:31-150: both endpoints store each
  // particle-particle bond, in file order.
  std::vector<int> pc(np, 0), po(np, 0), fc(np, 0), fo(np, 0), tmp(np, 0);
  for (int64_t b = 0; b < nbonds; ++b) {
    pc[bi[b]]++;
    pc[bj[b]]++;
  }
  for (int64_t b = 0; b < nfixed; ++b) fc[fi[b]]++;
  for (int i = 1; i < np; ++i) {
    po[i] = po[i - 1] + pc[i - 1];
    fo[i] = fo[i - 1] + fc[i - 1];
  }
  std::vector<int> idx(2 * nbonds);
  std::vector<double> kk(2 * nbonds), rr(2 * nbonds);
  for (int64_t b = 0; b < nbonds; ++b) {
    int i1 = bi[b], i2 = bj[b];
    int p1 = po[i1] + tmp[i1]++, p2 = po[i2] + tmp[i2]++;
    idx[p1] = i2;
    kk[p1] = k[b];
    rr[p1] = r0[b];
    idx[p2] = i1;
    kk[p2] = k[b];
    rr[p2] = r0[b];
  }
  std::fill(tmp.begin(), tmp.end(), 0);
  std::vector<double> fkk(nfixed), frr(nfixed), fxx(3 * nfixed);
  for (int64_t b = 0; b < nfixed; ++b) {
    int i1 = fi[b];
    int p = fo[i1] + tmp[i1]++;
    fkk[p] = fk[b];
    frr[p] = fr0[b];
    fxx[3 * p] = fxyz[3 * b];
    fxx[3 * p + 1] = fxyz[3 * b + 1];
    fxx[3 * p + 2] = fxyz[3 * b + 2];
  }
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  cudaFree(h->bpp_idx);
  cudaFree(h->bpp_k);
  cudaFree(h->bpp_r0);
  cudaFree(h->bfp_k);
  cudaFree(h->bfp_r0);
  cudaFree(h->bfp_xyz);
  h->bpp_idx = nullptr;
  h->bpp_k = h->bpp_r0 = h->bfp_k = h->bfp_r0 = h->bfp_xyz = nullptr;
  FSL_CUDA(dalloc(&h->bpp_idx, 2 * nbonds));
  FSL_CUDA(dalloc(&h->bpp_k, 2 * nbonds));
  FSL_CUDA(dalloc(&h->bpp_r0, 2 * nbonds));
  FSL_CUDA(dalloc(&h->bfp_k, nfixed));
  FSL_CUDA(dalloc(&h->bfp_r0, nfixed));
  FSL_CUDA(dalloc(&h->bfp_xyz, 3 * nfixed));
  if (np > 0) {
    FSL_CUDA(cudaMemcpy(h->bpp_cnt, pc.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bpp_off, po.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bfp_cnt, fc.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bfp_off, fo.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
  }
  if (nbonds > 0) {
    FSL_CUDA(cudaMemcpy(h->bpp_idx, idx.data(), sizeof(int) * 2 * nbonds, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bpp_k, kk.data(), sizeof(double) * 2 * nbonds, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bpp_r0, rr.data(), sizeof(double) * 2 * nbonds, cudaMemcpyHostToDevice));
  }
  if (nfixed > 0) {
    FSL_CUDA(cudaMemcpy(h->bfp_k, fkk.data(), sizeof(double) * nfixed, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bfp_r0, frr.data(), sizeof(double) * nfixed, cudaMemcpyHostToDevice));
    FSL_CUDA(cudaMemcpy(h->bfp_xyz, fxx.data(), sizeof(double) * 3 * nfixed, cudaMemcpyHostToDevice));
  }
  h->P.bonded = (nbonds + nfixed) > 0;
  drop_graph(h);  // the captured graph holds the old parameters
  return FSL_OK;
}

int fsl_set_graph(fsl_handle* h, int enable) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  h->use_graph = enable != 0;
  return FSL_OK;
}

int fsl_step(fsl_handle* h, int64_t nsteps) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  if (nsteps < 0) return set_error(FSL_E_ARG, "negative step count");
  FSL_CUDA(cudaSetDevice(h->device));
  for (int64_t k = 0; k < nsteps; ++k) {
    if (h->use_graph && h->steps > 0) {
      if (!h->gexec) {
        FSL_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(h);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (e != cudaSuccess) return set_error(FSL_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
        h->graph = g;
        FSL_CUDA(cudaGraphInstantiate(&h->gexec, g, 0));
      }
      FSL_CUDA(cudaGraphLaunch(h->gexec, h->stream));
    } else {
      enqueue_step(h);
      int rc = check_launch();
      if (rc) return rc;
    }
    h->steps++;
    int rc = prof_collect(h);
    if (rc) return rc;
  }
  return FSL_OK;
}

int fsl_profile(fsl_handle* h, int enable) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  // re-capture with or without the marks; a kept graph keeps its marks, so
  // the mark count of the last enqueued step stays valid
  if ((enable != 0) != h->prof.on) drop_graph(h);
  h->prof.on = enable != 0;
  h->stage_acc.clear();
  return FSL_OK;
}

int fsl_profile_read(fsl_handle* h, fsl_stage_time* out, int32_t max, int32_t* n) {
  if (!h || !n) return set_error(FSL_E_ARG, "null argument");
  int32_t k = 0;
  for (const auto& kv : h->stage_acc) {
    if (k < max && out) {
      std::memset(&out[k], 0, sizeof(fsl_stage_time));
      std::strncpy(out[k].name, kv.first.c_str(), sizeof(out[k].name) - 1);
      out[k].launches = kv.second.first;
      out[k].total_ms = kv.second.second;
    }
    ++k;
  }
  *n = k;
  return FSL_OK;
}

int fsl_sync(fsl_handle* h) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  int e[4];
  FSL_CUDA(cudaMemcpy(e, h->err, sizeof(e), cudaMemcpyDeviceToHost));
  if (e[fsl::ERR_ANY])
    return set_error(FSL_E_KERNEL, "kernel error word set: bits 0x%x", e[fsl::ERR_BITS]);
  return FSL_OK;
}

int fsl_get_positions(fsl_handle* h, double* out) {
  if (!h || !out) return set_error(FSL_E_ARG, "null argument");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemcpyAsync(out, h->q, sizeof(double) * 3 * (size_t)h->P.np, cudaMemcpyDeviceToHost,
                           h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

int fsl_set_positions(fsl_handle* h, const double* in) {
  if (!h || !in) return set_error(FSL_E_ARG, "null argument");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemcpyAsync(h->q, in, sizeof(double) * 3 * (size_t)h->P.np, cudaMemcpyHostToDevice,
                           h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

int fsl_get_forces(fsl_handle* h, double* out) {
  if (!h || !out) return set_error(FSL_E_ARG, "null argument");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemcpyAsync(out, h->F, sizeof(double) * 3 * (size_t)h->P.np, cudaMemcpyDeviceToHost,
                           h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

int fsl_get_velocity(fsl_handle* h, float* out) {
  if (!h || !out) return set_error(FSL_E_ARG, "null argument");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemcpyAsync(out, h->v, sizeof(float) * 3 * (size_t)h->P.nc, cudaMemcpyDeviceToHost,
                           h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

int fsl_get_status(fsl_handle* h, fsl_status* st) {
  if (!h || !st) return set_error(FSL_E_ARG, "null argument");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  int e[4];
  uint64_t t = 0;
  FSL_CUDA(cudaMemcpy(e, h->err, sizeof(e), cudaMemcpyDeviceToHost));
  FSL_CUDA(cudaMemcpy(&t, h->t_dev, sizeof(t), cudaMemcpyDeviceToHost));
  std::memset(st, 0, sizeof(*st));
  st->step = t;
  st->error_bits = e[fsl::ERR_BITS];
  st->np = h->P.np;
  st->nc = h->P.nc;
  st->graph = h->gexec != nullptr;
  st->launches_per_step = h->launches_per_step;
  return FSL_OK;
}

int fsl_set_step(fsl_handle* h, uint64_t step) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemcpyAsync(h->t_dev, &step, sizeof(step), cudaMemcpyHostToDevice, h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

int fsl_clear_errors(fsl_handle* h) {
  if (!h) return set_error(FSL_E_ARG, "null handle");
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemsetAsync(h->err, 0, sizeof(int) * 4, h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

// ------------------------------------------------- component entry points --
int fsl_neighbor_grid(fsl_handle* h, int32_t* dims3) {
  if (!h || !dims3) return set_error(FSL_E_ARG, "null argument");
  dims3[0] = h->P.mnx;
  dims3[1] = h->P.mny;
  dims3[2] = h->P.mnz;
  return FSL_OK;
}

int fsl_cell_list(fsl_handle* h, int32_t* cell_of, int32_t* start, int32_t* sorted) {
  if (!h || !cell_of || !start || !sorted) return set_error(FSL_E_ARG, "null argument");
  const fsl::Params& P = h->P;
  FSL_CUDA(cudaSetDevice(h->device));
  fsl::launch_cells(P, h->q, h->cell_of, h->cnt, h->start, h->fill, h->tmp, h->sorted, h->bsum, h->err,
                    h->stream);
  int rc = check_launch();
  if (rc) return rc;
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  if (P.np > 0) {
    FSL_CUDA(cudaMemcpy(cell_of, h->cell_of, sizeof(int) * P.np, cudaMemcpyDeviceToHost));
    FSL_CUDA(cudaMemcpy(sorted, h->sorted, sizeof(int) * P.np, cudaMemcpyDeviceToHost));
  }
  FSL_CUDA(cudaMemcpy(start, h->start, sizeof(int) * ((size_t)P.mN + 1), cudaMemcpyDeviceToHost));
  return FSL_OK;
}

int fsl_compute_forces(fsl_handle* h, double* F) {
  if (!h || !F) return set_error(FSL_E_ARG, "null argument");
  FSL_CUDA(cudaSetDevice(h->device));
  enqueue_cells_forces(h, h->q);
  int rc = check_launch();
  if (rc) return rc;
  return fsl_get_forces(h, F);
}

int fsl_spread(fsl_handle* h, const double* F, double* f) {
  if (!h || !F || !f) return set_error(FSL_E_ARG, "null argument");
  const fsl::Params& P = h->P;
  FSL_CUDA(cudaSetDevice(h->device));
  FSL_CUDA(cudaMemcpyAsync(h->F, F, sizeof(double) * 3 * (size_t)P.np, cudaMemcpyHostToDevice, h->stream));
  FSL_CUDA(cudaMemsetAsync(h->grid, 0, sizeof(unsigned long long) * 3 * (size_t)P.nc, h->stream));
  fsl::launch_spread(P, 0, nullptr, h->q, h->F, h->q, h->noise, h->grid, h->err, h->stream);
  int rc = check_launch();
  if (rc) return rc;
  std::vector<long long> g(3 * (size_t)P.nc);
  FSL_CUDA(cudaMemcpyAsync(g.data(), h->grid, sizeof(long long) * g.size(), cudaMemcpyDeviceToHost,
                           h->stream));
  // the step expects a cleared spread field
  FSL_CUDA(cudaMemsetAsync(h->grid, 0, sizeof(unsigned long long) * g.size(), h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  const double sc = fsl::kFixedInv / P.dV;
  for (size_t k = 0; k < g.size(); ++k) f[k] = (double)g[k] * sc;
  return FSL_OK;
}

int fsl_solve(fsl_handle* h, const double* W, double* v) {
  if (!h || !W || !v) return set_error(FSL_E_ARG, "null argument");
  const fsl::Params& P = h->P;
  const size_t n3 = 3 * (size_t)P.nc;
  FSL_CUDA(cudaSetDevice(h->device));
  if (!h->wext) FSL_CUDA(dalloc(&h->wext, n3));
  std::vector<float> w(n3);
  for (size_t k = 0; k < n3; ++k) w[k] = (float)W[k];
  FSL_CUDA(cudaMemcpyAsync(h->wext, w.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, h->stream));
  fsl::launch_solve(P, h->fft, nullptr, nullptr, 1, h->wext, h->wbuf, h->spec, h->v, h->stream);
  int rc = check_launch();
  if (rc) return rc;
  FSL_CUDA(cudaMemcpyAsync(w.data(), h->v, sizeof(float) * n3, cudaMemcpyDeviceToHost, h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  for (size_t k = 0; k < n3; ++k) v[k] = (double)w[k];
  return FSL_OK;
}

int fsl_interpolate(fsl_handle* h, const double* vin, double* u) {
  if (!h || !vin || !u) return set_error(FSL_E_ARG, "null argument");
  const fsl::Params& P = h->P;
  const size_t n3 = 3 * (size_t)P.nc;
  FSL_CUDA(cudaSetDevice(h->device));
  if (!h->u) FSL_CUDA(dalloc(&h->u, 3 * (size_t)P.np));
  std::vector<float> w(n3);
  for (size_t k = 0; k < n3; ++k) w[k] = (float)vin[k];
  FSL_CUDA(cudaMemcpyAsync(h->v, w.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, h->stream));
  fsl::launch_interp(P, h->q, h->v, h->u, h->stream);
  int rc = check_launch();
  if (rc) return rc;
  FSL_CUDA(cudaMemcpyAsync(u, h->u, sizeof(double) * 3 * (size_t)P.np, cudaMemcpyDeviceToHost, h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

int fsl_noise(fsl_handle* h, uint64_t t, uint64_t first, int64_t count, float* out) {
  if (!h || !out || count < 0) return set_error(FSL_E_ARG, "bad argument");
  FSL_CUDA(cudaSetDevice(h->device));
  if (count > h->nbuf_n) {
    cudaFree(h->nbuf);
    h->nbuf = nullptr;
    h->nbuf_n = 0;
    FSL_CUDA(dalloc(&h->nbuf, count));
    h->nbuf_n = count;
  }
  fsl::launch_noise_range(h->P, t, first, count, h->nbuf, h->stream);
  int rc = check_launch();
  if (rc) return rc;
  FSL_CUDA(cudaMemcpyAsync(out, h->nbuf, sizeof(float) * count, cudaMemcpyDeviceToHost, h->stream));
  FSL_CUDA(cudaStreamSynchronize(h->stream));
  return FSL_OK;
}

}  // extern "C"
