// fsl_api.cu -- the single-instance C ABI of libfluamsl (include/fluamsl.h):
// a handle is one slot in a one-instance group, stepped by its own Exec (a
// CUDA graph of the step), plus the component entry points.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fsl_group.cuh"

struct fsl_handle {
  fsl_config cfg{};
  fsl::Slot slot;
  fsl::Group group;
  fsl::Exec exec;
  float* nbuf = nullptr;  // scratch of fsl_noise
  int64_t nbuf_n = 0;
};

namespace {

using fsl::errorf;

void free_handle(fsl_handle* h) {
  if (!h) return;
  if (h->exec.stream) cudaStreamSynchronize(h->exec.stream);
  if (h->nbuf) cudaFree(h->nbuf);
  fsl::exec_destroy(h->exec);
  fsl::group_destroy(h->group);
  fsl::slot_free(h->slot);
  delete h;
}

// The instance table must be current before any launch outside fsl_step.
int prepare(fsl_handle* h) {
  FSL_TRY(cudaSetDevice(h->exec.device));
  h->group.stream = h->exec.stream;
  return fsl::group_upload(h->group);
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fsl::cuda_fail(e, "kernel launch");
  return FSL_OK;
}

const fsl::Params& params(const fsl_handle* h) { return h->slot.r.P; }
const fsl::Rep& rep(const fsl_handle* h) { return h->slot.r; }

// The stage entry points exchange the FP32 fields of the default form.
int fixed_form_only(const fsl_handle* h, const char* what) {
  if (params(h).prec == fsl::PREC_FIXED) return FSL_OK;
  return errorf(FSL_E_ARG, "%s: available in the FIXED64 precision form only", what);
}

}  // namespace

extern "C" {

const char* fsl_last_error(void) { return fsl::last_error(); }

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
  // src/loadDataMain.cu:260-272
  c->radius = 1.0;
  c->ndrift = 1;
  c->use_rfd = 1;
  c->density = 1.0;
}

int fsl_create(const fsl_config* cfg, int64_t np, const double* q, fsl_handle** out) {
  if (!cfg || !out) return errorf(FSL_E_ARG, "null argument");
  *out = nullptr;
  fsl::Params P;
  int rc = fsl::make_params(*cfg, np, P);
  if (rc) return rc;
  if (np > 0 && !q) return errorf(FSL_E_ARG, "null positions");
  int dev = cfg->device;
  if (dev < 0) FSL_TRY(cudaGetDevice(&dev));
  fsl_handle* h = new fsl_handle();
  h->cfg = *cfg;
  auto fail = [&](int code) {
    free_handle(h);
    return code;
  };
  if ((rc = fsl::exec_init(h->exec, dev))) return fail(rc);
  if ((rc = fsl::slot_alloc(h->slot, P, (int)np, h->exec.stream))) return fail(rc);
  if ((rc = fsl::slot_reset(h->slot, P, q, *cfg, h->exec.stream))) return fail(rc);
  if ((rc = fsl::group_init(h->group, P))) return fail(rc);
  h->group.slots.push_back(&h->slot);
  h->exec.groups.push_back(&h->group);
  if ((rc = prepare(h))) return fail(rc);
  cudaError_t e = cudaStreamSynchronize(h->exec.stream);
  if (e != cudaSuccess) return fail(fsl::cuda_fail(e, "create"));
  *out = h;
  return FSL_OK;
}

void fsl_destroy(fsl_handle* h) {
  if (!h) return;
  cudaSetDevice(h->exec.device);
  free_handle(h);
}

void* fsl_stream(fsl_handle* h) { return h ? (void*)h->exec.stream : nullptr; }

int fsl_load_bonds(fsl_handle* h, int64_t nbonds, const int32_t* bi, const int32_t* bj,
                   const double* k, const double* r0, int64_t nfixed, const int32_t* fi,
                   const double* fk, const double* fr0, const double* fxyz) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  FSL_TRY(cudaSetDevice(h->exec.device));
  int rc = fsl::slot_bonds(h->slot, nbonds, bi, bj, k, r0, nfixed, fi, fk, fr0, fxyz, h->exec.stream);
  h->group.dirty = true;  // new table pointers and the bonded flag
  return rc;
}

int fsl_load_bonds_directed(fsl_handle* h, int64_t nentries, const int32_t* bi, const int32_t* bj,
                            const double* k, const double* r0, int64_t nfixed, const int32_t* fi,
                            const double* fk, const double* fr0, const double* fxyz) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  FSL_TRY(cudaSetDevice(h->exec.device));
  int rc = fsl::slot_bonds(h->slot, nentries, bi, bj, k, r0, nfixed, fi, fk, fr0, fxyz, h->exec.stream,
                           true);
  h->group.dirty = true;
  return rc;
}

int fsl_set_graph(fsl_handle* h, int enable) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  h->exec.use_graph = enable != 0;
  return FSL_OK;
}

int fsl_step(fsl_handle* h, int64_t nsteps) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  return fsl::exec_step(h->exec, nsteps);
}

int fsl_profile(fsl_handle* h, int enable) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  // the graph is captured again with or without the marks; a kept graph
  // keeps its marks, so the mark count of the last enqueued step stays valid
  h->group.prof.on = enable != 0;
  h->group.stage_acc.clear();
  return FSL_OK;
}

int fsl_profile_read(fsl_handle* h, fsl_stage_time* out, int32_t max, int32_t* n) {
  if (!h || !n) return errorf(FSL_E_ARG, "null argument");
  int32_t k = 0;
  for (const auto& kv : h->group.stage_acc) {
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
  if (!h) return errorf(FSL_E_ARG, "null handle");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  int e[4];
  FSL_TRY(cudaMemcpy(e, rep(h).err, sizeof(e), cudaMemcpyDeviceToHost));
  if (e[fsl::ERR_ANY]) return errorf(FSL_E_KERNEL, "kernel error word set: bits 0x%x", e[fsl::ERR_BITS]);
  return FSL_OK;
}

int fsl_get_positions(fsl_handle* h, double* out) {
  if (!h || !out) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaMemcpyAsync(out, rep(h).q, sizeof(double) * 3 * (size_t)params(h).np,
                          cudaMemcpyDeviceToHost, h->exec.stream));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_set_positions(fsl_handle* h, const double* in) {
  if (!h || !in) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaMemcpyAsync(rep(h).q, in, sizeof(double) * 3 * (size_t)params(h).np,
                          cudaMemcpyHostToDevice, h->exec.stream));
  if (int rc = fsl::slot_mark_moved(h->slot, h->exec.stream)) return rc;
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_step_io(fsl_handle* h, const double* in, double* out) {
  if (!h || !in || !out) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  if (!fsl::pinned_host(in) || !fsl::pinned_host(out)) {
    // pageable buffers: the copies stay outside the step's graph
    if (int rc = fsl_set_positions(h, in)) return rc;
    if (int rc = fsl_step(h, 1)) return rc;
    return fsl_get_positions(h, out);
  }
  fsl::Group& g = h->group;
  g.io_in = in;
  g.io_out = out;
  g.io_bytes = sizeof(double) * 3 * (size_t)params(h).np;
  const int rc = fsl::exec_step(h->exec, 1);
  g.io_in = nullptr;
  g.io_out = nullptr;
  if (rc) return rc;
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_get_forces(fsl_handle* h, double* out) {
  if (!h || !out) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaMemcpyAsync(out, rep(h).F, sizeof(double) * 3 * (size_t)params(h).np,
                          cudaMemcpyDeviceToHost, h->exec.stream));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_get_velocity(fsl_handle* h, float* out) {
  if (!h || !out) return errorf(FSL_E_ARG, "null argument");
  if (params(h).prec == fsl::PREC_F64)
    return errorf(FSL_E_ARG, "fsl_get_velocity: the FP64 form's field is read by fsl_get_velocity_f64");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaMemcpyAsync(out, rep(h).v, sizeof(float) * 3 * (size_t)params(h).nc,
                          cudaMemcpyDeviceToHost, h->exec.stream));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_get_velocity_f64(fsl_handle* h, double* out) {
  if (!h || !out) return errorf(FSL_E_ARG, "null argument");
  const size_t n3 = 3 * (size_t)params(h).nc;
  if (params(h).prec != fsl::PREC_F64) {
    std::vector<float> v(n3);
    int rc = fsl_get_velocity(h, v.data());
    if (rc) return rc;
    for (size_t k = 0; k < n3; ++k) out[k] = (double)v[k];
    return FSL_OK;
  }
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaMemcpyAsync(out, rep(h).v64, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->exec.stream));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_set_velocity_f64(fsl_handle* h, const double* in) {
  if (!h || !in) return errorf(FSL_E_ARG, "null argument");
  if (params(h).scheme != FSL_SCHEME_INCOMPRESSIBLE)
    return errorf(FSL_E_ARG, "fsl_set_velocity_f64: the incompressible scheme only");
  int rc = prepare(h);
  if (rc) return rc;
  const fsl::Batch& B = h->group.B;
  cudaStream_t s = h->exec.stream;
  FSL_TRY(cudaMemcpyAsync(rep(h).v64, in, sizeof(double) * 3 * (size_t)params(h).nc,
                          cudaMemcpyHostToDevice, s));
  // src/runSchemeIncompressible.cu:82-96: the projection of the initial field
  fsl::launch_inc_load(B, s);
  fsl::launch_fft64_3d(B, -1, 0, s);
  fsl::launch_inc_fourier(B, 0, s);
  fsl::launch_fft64_3d(B, +1, 1, s);
  if ((rc = check_launch())) return rc;
  FSL_TRY(cudaStreamSynchronize(s));
  return FSL_OK;
}

int fsl_get_tuning(fsl_handle* h, fsl_class_tuning* out) {
  if (!h || !out) return errorf(FSL_E_ARG, "null argument");
  fsl::group_tuning(h->group, out);
  return FSL_OK;
}

int fsl_get_status(fsl_handle* h, fsl_status* st) {
  if (!h || !st) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  int e[4];
  uint64_t t = 0;
  FSL_TRY(cudaMemcpy(e, rep(h).err, sizeof(e), cudaMemcpyDeviceToHost));
  FSL_TRY(cudaMemcpy(&t, rep(h).t, sizeof(t), cudaMemcpyDeviceToHost));
  std::memset(st, 0, sizeof(*st));
  st->step = t;
  st->error_bits = e[fsl::ERR_BITS];
  st->np = params(h).np;
  st->nc = params(h).nc;
  st->graph = h->exec.gexec != nullptr;
  st->launches_per_step = h->exec.launches_per_step;
  return FSL_OK;
}

int fsl_get_observables(fsl_handle* h, fsl_observables* out) {
  if (!h || !out) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  return fsl::slot_read_observables(h->slot, h->exec.stream, out);
}

int fsl_reset_observables(fsl_handle* h) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  if (!params(h).observe) return errorf(FSL_E_ARG, "observables are off (fsl_config.observables = 0)");
  FSL_TRY(cudaSetDevice(h->exec.device));
  return fsl::slot_reset_observables(h->slot, h->exec.stream);
}

int fsl_set_step(fsl_handle* h, uint64_t step) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  FSL_TRY(cudaSetDevice(h->exec.device));
  FSL_TRY(cudaMemcpyAsync(rep(h).t, &step, sizeof(step), cudaMemcpyHostToDevice, h->exec.stream));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

int fsl_clear_errors(fsl_handle* h) {
  if (!h) return errorf(FSL_E_ARG, "null handle");
  FSL_TRY(cudaSetDevice(h->exec.device));
  if (int rc = fsl::slot_clear_errors(h->slot, h->exec.stream)) return rc;
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

// ------------------------------------------------- component entry points --
int fsl_neighbor_grid(fsl_handle* h, int32_t* dims3) {
  if (!h || !dims3) return errorf(FSL_E_ARG, "null argument");
  dims3[0] = params(h).mnx;
  dims3[1] = params(h).mny;
  dims3[2] = params(h).mnz;
  return FSL_OK;
}

int fsl_cell_list(fsl_handle* h, int32_t* cell_of, int32_t* start, int32_t* sorted) {
  if (!h || !cell_of || !start || !sorted) return errorf(FSL_E_ARG, "null argument");
  int rc = prepare(h);
  if (rc) return rc;
  const fsl::Params& P = params(h);
  if ((rc = fsl::slot_request_lists(h->slot, h->exec.stream))) return rc;
  fsl::launch_cells(h->group.B, 0, h->exec.stream);
  if ((rc = check_launch())) return rc;
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  if (P.np > 0) {
    FSL_TRY(cudaMemcpy(cell_of, rep(h).cell_of, sizeof(int) * P.np, cudaMemcpyDeviceToHost));
    FSL_TRY(cudaMemcpy(sorted, rep(h).sorted, sizeof(int) * P.np, cudaMemcpyDeviceToHost));
  }
  FSL_TRY(cudaMemcpy(start, rep(h).start, sizeof(int) * ((size_t)P.mN + 1), cudaMemcpyDeviceToHost));
  return FSL_OK;
}

int fsl_compute_forces(fsl_handle* h, double* F) {
  if (!h || !F) return errorf(FSL_E_ARG, "null argument");
  int rc = prepare(h);
  if (rc) return rc;
  if ((rc = fsl::slot_request_lists(h->slot, h->exec.stream))) return rc;
  fsl::launch_pair_lists(h->group.B, 0, h->exec.stream);
  fsl::launch_forces(h->group.B, 0, h->exec.stream);
  if ((rc = check_launch())) return rc;
  return fsl_get_forces(h, F);
}

int fsl_spread(fsl_handle* h, const double* F, double* f) {
  if (!h || !F || !f) return errorf(FSL_E_ARG, "null argument");
  int rc = fixed_form_only(h, "fsl_spread");
  if (rc) return rc;
  rc = prepare(h);
  if (rc) return rc;
  const fsl::Params& P = params(h);
  const fsl::Rep& R = rep(h);
  cudaStream_t s = h->exec.stream;
  FSL_TRY(cudaMemcpyAsync(R.F, F, sizeof(double) * 3 * (size_t)P.np, cudaMemcpyHostToDevice, s));
  FSL_TRY(cudaMemsetAsync(R.grid, 0, sizeof(unsigned long long) * 3 * (size_t)P.nc, s));
  fsl::launch_spread(h->group.B, 0, 0, s);
  if ((rc = check_launch())) return rc;
  std::vector<long long> g(3 * (size_t)P.nc);
  FSL_TRY(cudaMemcpyAsync(g.data(), R.grid, sizeof(long long) * g.size(), cudaMemcpyDeviceToHost, s));
  // the step expects a cleared spread field
  FSL_TRY(cudaMemsetAsync(R.grid, 0, sizeof(unsigned long long) * g.size(), s));
  FSL_TRY(cudaStreamSynchronize(s));
  const double sc = fsl::kFixedInv / P.dV;
  for (size_t k = 0; k < g.size(); ++k) f[k] = (double)g[k] * sc;
  return FSL_OK;
}

int fsl_solve(fsl_handle* h, const double* W, double* v) {
  if (!h || !W || !v) return errorf(FSL_E_ARG, "null argument");
  int rc = fixed_form_only(h, "fsl_solve");
  if (rc) return rc;
  rc = prepare(h);
  if (rc) return rc;
  const fsl::Params& P = params(h);
  const fsl::Rep& R = rep(h);
  cudaStream_t s = h->exec.stream;
  const size_t n3 = 3 * (size_t)P.nc;
  std::vector<float> w(n3);
  for (size_t k = 0; k < n3; ++k) w[k] = (float)W[k];
  FSL_TRY(cudaMemcpyAsync(R.wbuf, w.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, s));
  fsl::launch_solve(h->group.B, h->group.fft, 1, 1.0, 1, s);
  if ((rc = check_launch())) return rc;
  FSL_TRY(cudaMemcpyAsync(w.data(), R.v, sizeof(float) * n3, cudaMemcpyDeviceToHost, s));
  FSL_TRY(cudaStreamSynchronize(s));
  for (size_t k = 0; k < n3; ++k) v[k] = (double)w[k];
  return FSL_OK;
}

int fsl_interpolate(fsl_handle* h, const double* vin, double* u) {
  if (!h || !vin || !u) return errorf(FSL_E_ARG, "null argument");
  int rc = fixed_form_only(h, "fsl_interpolate");
  if (rc) return rc;
  rc = prepare(h);
  if (rc) return rc;
  const fsl::Params& P = params(h);
  const fsl::Rep& R = rep(h);
  cudaStream_t s = h->exec.stream;
  const size_t n3 = 3 * (size_t)P.nc;
  std::vector<float> w(n3);
  for (size_t k = 0; k < n3; ++k) w[k] = (float)vin[k];
  FSL_TRY(cudaMemcpyAsync(R.v, w.data(), sizeof(float) * n3, cudaMemcpyHostToDevice, s));
  fsl::launch_interp(h->group.B, s);
  if ((rc = check_launch())) return rc;
  FSL_TRY(cudaMemcpyAsync(u, R.u, sizeof(double) * 3 * (size_t)P.np, cudaMemcpyDeviceToHost, s));
  FSL_TRY(cudaStreamSynchronize(s));
  return FSL_OK;
}

int fsl_noise(fsl_handle* h, uint64_t t, uint64_t first, int64_t count, float* out) {
  if (!h || !out || count < 0) return errorf(FSL_E_ARG, "bad argument");
  FSL_TRY(cudaSetDevice(h->exec.device));
  if (count > h->nbuf_n) {
    cudaFree(h->nbuf);
    h->nbuf = nullptr;
    h->nbuf_n = 0;
    FSL_TRY(cudaMalloc((void**)&h->nbuf, sizeof(float) * std::max<int64_t>(count, 1)));
    h->nbuf_n = count;
  }
  fsl::launch_noise_range(params(h), t, first, count, h->nbuf, h->exec.stream);
  int rc = check_launch();
  if (rc) return rc;
  FSL_TRY(cudaMemcpyAsync(out, h->nbuf, sizeof(float) * count, cudaMemcpyDeviceToHost, h->exec.stream));
  FSL_TRY(cudaStreamSynchronize(h->exec.stream));
  return FSL_OK;
}

}  // extern "C"
