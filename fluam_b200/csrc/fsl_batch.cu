// fsl_batch.cu -- batched instances (the fsl_batch_* C ABI): one slot per
// instance, instances grouped by size class, every class stepped by one
// launch per stage on its own stream, the whole step captured in one graph.
#include <algorithm>
#include <cstring>
#include <iterator>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "fsl_group.cuh"

namespace {

// Where instance i's particles sit in the packed arrays.
struct PackEnt {
  double* q;
  int* err;
  long long off;  // first double of the instance in the packed array
  int np;
  int pad;
  uint64_t* vl_flag;  // Verlet list: rebuild word, reference positions,
  const double* qref;  // (skin / 2)^2 and the step counter (null qref: no list)
  double vl_half2;
  const uint64_t* t;
};

// dir = 0: packed <- q of every instance; dir = 1: q <- packed.
// Block row blockIdx.y is the instance.
__global__ void k_pack(const PackEnt* __restrict__ ents, double* __restrict__ packed, int dir) {
  const PackEnt e = ents[blockIdx.y];
  const long long n3 = 3ll * e.np;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n3;
       k += (long long)gridDim.x * blockDim.x) {
    if (dir == 0) packed[e.off + k] = e.q[k];
    else e.q[k] = packed[e.off + k];
  }
  // new positions: the Verlet list is rebuilt at the next evaluation at q
  // if a particle left its skin (as k_moved_check)
  if (dir == 1 && e.qref) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < e.np;
         i += (long long)gridDim.x * blockDim.x) {
      double d2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double v = packed[e.off + d * (long long)e.np + i] - e.qref[d * (long long)e.np + i];
        d2 += v * v;
      }
      if (d2 > e.vl_half2) e.vl_flag[0] = *e.t + 1;
    }
  }
}

// errs[i] = error bits of instance i with bit 30 set, or 0 if its word is clear
__global__ void k_gather_err(const PackEnt* __restrict__ ents, int n, int* __restrict__ errs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int* w = ents[i].err;
    errs[i] = w[fsl::ERR_ANY] ? (w[fsl::ERR_BITS] | 0x40000000) : 0;
  }
}

}  // namespace

struct fsl_batch {
  std::vector<std::unique_ptr<fsl::Slot>> slots;  // instance order
  std::map<fsl::ClassKey, std::unique_ptr<fsl::Group>> groups;
  fsl::Exec exec;
  PackEnt* d_ents = nullptr;
  double* d_packed = nullptr;
  int* d_errs = nullptr;
  long long packed_n = 0;
  int max_np = 0;
  int64_t nc_total = 0;
};

namespace {

using fsl::errorf;

// Prefixes the current message with the instance index.
int instance_error(int code, int i) {
  std::string m = fsl::last_error();
  return errorf(code, "instance %d: %s", i, m.c_str());
}

void free_batch(fsl_batch* b) {
  if (!b) return;
  if (b->exec.stream) cudaStreamSynchronize(b->exec.stream);
  fsl::exec_destroy(b->exec);
  for (auto& kv : b->groups) fsl::group_destroy(*kv.second);
  for (auto& s : b->slots) fsl::slot_free(*s);
  cudaFree(b->d_ents);
  cudaFree(b->d_packed);
  cudaFree(b->d_errs);
  delete b;
}

int check_index(const fsl_batch* b, int32_t i) {
  if (!b) return errorf(FSL_E_ARG, "null batch");
  if (i < 0 || i >= (int32_t)b->slots.size()) return errorf(FSL_E_ARG, "instance %d out of range", i);
  return FSL_OK;
}

void pack_on(fsl_batch* b, int dir, cudaStream_t st) {
  if (b->slots.empty() || b->max_np == 0) return;
  unsigned bx = (unsigned)std::min<long long>((3ll * b->max_np + 255) / 256, 64);
  k_pack<<<dim3(bx, (unsigned)b->slots.size()), 256, 0, st>>>(b->d_ents, b->d_packed, dir);
}

int pack(fsl_batch* b, int dir) {
  pack_on(b, dir, b->exec.stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fsl::cuda_fail(e, "pack kernel");
  return FSL_OK;
}

}  // namespace

extern "C" {

int fsl_batch_create(int32_t n, const fsl_config* cfgs, const int64_t* np, const double* const* q,
                     fsl_batch** out) {
  if (!out) return errorf(FSL_E_ARG, "null argument");
  *out = nullptr;
  if (n < 0 || (n > 0 && (!cfgs || !np || !q))) return errorf(FSL_E_ARG, "bad instance arrays");
  std::vector<fsl::Params> P(n);
  int dev = -1;
  for (int32_t i = 0; i < n; ++i) {
    int rc = fsl::make_params(cfgs[i], np[i], P[i]);
    if (rc) return instance_error(rc, i);
    if (np[i] > 0 && !q[i]) return errorf(FSL_E_ARG, "instance %d: null positions", i);
    if (cfgs[i].device >= 0) {
      if (dev >= 0 && dev != cfgs[i].device)
        return errorf(FSL_E_ARG, "instance %d: all instances of a batch share one device", i);
      dev = cfgs[i].device;
    }
  }
  if (dev < 0) FSL_TRY(cudaGetDevice(&dev));
  fsl_batch* b = new fsl_batch();
  auto fail = [&](int code) {
    free_batch(b);
    return code;
  };
  int rc = fsl::exec_init(b->exec, dev);
  if (rc) return fail(rc);
  cudaStream_t st = b->exec.stream;
  std::vector<PackEnt> ents(n);
  long long off = 0;
  for (int32_t i = 0; i < n; ++i) {
    b->slots.emplace_back(new fsl::Slot());
    fsl::Slot& s = *b->slots.back();
    if ((rc = fsl::slot_alloc(s, P[i], (int)np[i], st))) return fail(instance_error(rc, i));
    if ((rc = fsl::slot_reset(s, P[i], q[i], cfgs[i], st))) return fail(rc);
    fsl::ClassKey key = fsl::class_of(P[i]);
    auto it = b->groups.find(key);
    if (it == b->groups.end()) {
      std::unique_ptr<fsl::Group> g(new fsl::Group());
      if ((rc = fsl::group_init(*g, P[i]))) return fail(rc);
      it = b->groups.emplace(key, std::move(g)).first;
    }
    it->second->slots.push_back(&s);
    ents[i] = PackEnt{s.r.q, s.r.err, off, (int)np[i], 0, s.r.vl_flag, s.r.P.verlet ? s.r.qref : nullptr,
                      s.r.P.vl_half2, s.r.t};
    off += 3ll * np[i];
    b->max_np = std::max(b->max_np, (int)np[i]);
    b->nc_total += P[i].nc;
  }
  // the largest classes first: their streams start their work first
  std::vector<fsl::Group*> order;
  for (auto& kv : b->groups) order.push_back(kv.second.get());
  std::stable_sort(order.begin(), order.end(), [](const fsl::Group* a, const fsl::Group* c) {
    return (long long)a->P0.nc * a->slots.size() > (long long)c->P0.nc * c->slots.size();
  });
  b->exec.groups = order;
  b->packed_n = off;
  cudaError_t e;
  if ((e = cudaMalloc((void**)&b->d_ents, sizeof(PackEnt) * std::max(n, 1))) != cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_packed, sizeof(double) * std::max<long long>(off, 1))) != cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_errs, sizeof(int) * std::max(n, 1))) != cudaSuccess)
    return fail(fsl::cuda_fail(e, "batch tables"));
  if (n > 0 && (e = cudaMemcpyAsync(b->d_ents, ents.data(), sizeof(PackEnt) * n, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(fsl::cuda_fail(e, "batch tables"));
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(fsl::cuda_fail(e, "create"));
  *out = b;
  return FSL_OK;
}

void fsl_batch_destroy(fsl_batch* b) {
  if (!b) return;
  cudaSetDevice(b->exec.device);
  free_batch(b);
}

void* fsl_batch_stream(fsl_batch* b) { return b ? (void*)b->exec.stream : nullptr; }

int fsl_batch_load_bonds(fsl_batch* b, int32_t i, int64_t nbonds, const int32_t* bi,
                         const int32_t* bj, const double* k, const double* r0, int64_t nfixed,
                         const int32_t* fi, const double* fk, const double* fr0, const double* fxyz) {
  int rc = check_index(b, i);
  if (rc) return rc;
  FSL_TRY(cudaSetDevice(b->exec.device));
  fsl::Slot& s = *b->slots[i];
  // every stream of the batch may still read the old tables
  FSL_TRY(cudaDeviceSynchronize());
  rc = fsl::slot_bonds(s, nbonds, bi, bj, k, r0, nfixed, fi, fk, fr0, fxyz, b->exec.stream);
  b->groups[fsl::class_of(s.r.P)]->dirty = true;
  return rc;
}

int fsl_batch_step(fsl_batch* b, int64_t nsteps) {
  if (!b) return errorf(FSL_E_ARG, "null batch");
  return fsl::exec_step(b->exec, nsteps);
}

int fsl_batch_sync(fsl_batch* b) {
  if (!b) return errorf(FSL_E_ARG, "null batch");
  FSL_TRY(cudaSetDevice(b->exec.device));
  const int n = (int)b->slots.size();
  if (n == 0) return FSL_OK;
  k_gather_err<<<(n + 255) / 256, 256, 0, b->exec.stream>>>(b->d_ents, n, b->d_errs);
  FSL_TRY(cudaGetLastError());
  std::vector<int> errs(n);
  FSL_TRY(cudaMemcpyAsync(errs.data(), b->d_errs, sizeof(int) * n, cudaMemcpyDeviceToHost, b->exec.stream));
  FSL_TRY(cudaStreamSynchronize(b->exec.stream));
  for (int i = 0; i < n; ++i)
    if (errs[i])
      return errorf(FSL_E_KERNEL, "instance %d: kernel error word set: bits 0x%x", i, errs[i] & 0xffff);
  return FSL_OK;
}

int fsl_batch_get_positions(fsl_batch* b, int32_t i, double* out) {
  int rc = check_index(b, i);
  if (rc) return rc;
  if (!out) return errorf(FSL_E_ARG, "null argument");
  const fsl::Rep& r = b->slots[i]->r;
  FSL_TRY(cudaSetDevice(b->exec.device));
  FSL_TRY(cudaMemcpyAsync(out, r.q, sizeof(double) * 3 * (size_t)r.P.np, cudaMemcpyDeviceToHost,
                          b->exec.stream));
  FSL_TRY(cudaStreamSynchronize(b->exec.stream));
  return FSL_OK;
}

int fsl_batch_get_forces(fsl_batch* b, int32_t i, double* out) {
  int rc = check_index(b, i);
  if (rc) return rc;
  if (!out) return errorf(FSL_E_ARG, "null argument");
  const fsl::Rep& r = b->slots[i]->r;
  FSL_TRY(cudaSetDevice(b->exec.device));
  FSL_TRY(cudaMemcpyAsync(out, r.F, sizeof(double) * 3 * (size_t)r.P.np, cudaMemcpyDeviceToHost,
                          b->exec.stream));
  FSL_TRY(cudaStreamSynchronize(b->exec.stream));
  return FSL_OK;
}

int fsl_batch_get_status(fsl_batch* b, int32_t i, fsl_status* st) {
  int rc = check_index(b, i);
  if (rc) return rc;
  if (!st) return errorf(FSL_E_ARG, "null argument");
  const fsl::Rep& r = b->slots[i]->r;
  FSL_TRY(cudaSetDevice(b->exec.device));
  FSL_TRY(cudaStreamSynchronize(b->exec.stream));
  int e[4];
  uint64_t t = 0;
  FSL_TRY(cudaMemcpy(e, r.err, sizeof(e), cudaMemcpyDeviceToHost));
  FSL_TRY(cudaMemcpy(&t, r.t, sizeof(t), cudaMemcpyDeviceToHost));
  std::memset(st, 0, sizeof(*st));
  st->step = t;
  st->error_bits = e[fsl::ERR_BITS];
  st->np = r.P.np;
  st->nc = r.P.nc;
  st->graph = b->exec.gexec != nullptr;
  st->launches_per_step = b->exec.launches_per_step;
  return FSL_OK;
}

int fsl_batch_get_observables(fsl_batch* b, int32_t i, fsl_observables* out) {
  int rc = check_index(b, i);
  if (rc) return rc;
  if (!out) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(b->exec.device));
  return fsl::slot_read_observables(*b->slots[i], b->exec.stream, out);
}

int fsl_batch_reset_observables(fsl_batch* b, int32_t i) {
  int rc = check_index(b, i);
  if (rc) return rc;
  if (!b->slots[i]->r.P.observe) return errorf(FSL_E_ARG, "instance %d: observables are off", i);
  FSL_TRY(cudaSetDevice(b->exec.device));
  return fsl::slot_reset_observables(*b->slots[i], b->exec.stream);
}

int fsl_batch_get_positions_packed_async(fsl_batch* b, double* host) {
  if (!b || !host) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(b->exec.device));
  int rc = pack(b, 0);
  if (rc) return rc;
  if (b->packed_n > 0)
    FSL_TRY(cudaMemcpyAsync(host, b->d_packed, sizeof(double) * b->packed_n, cudaMemcpyDeviceToHost,
                            b->exec.stream));
  return FSL_OK;
}

int fsl_batch_set_positions_packed_async(fsl_batch* b, const double* host) {
  if (!b || !host) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(b->exec.device));
  if (b->packed_n > 0)
    FSL_TRY(cudaMemcpyAsync(b->d_packed, host, sizeof(double) * b->packed_n, cudaMemcpyHostToDevice,
                            b->exec.stream));
  return pack(b, 1);
}

int fsl_batch_step_io(fsl_batch* b, const double* in, double* out) {
  if (!b || !in || !out) return errorf(FSL_E_ARG, "null argument");
  FSL_TRY(cudaSetDevice(b->exec.device));
  if (!fsl::pinned_host(in) || !fsl::pinned_host(out)) {
    // pageable buffers: the copies stay outside the step's graph
    if (int rc = fsl_batch_set_positions_packed(b, in)) return rc;
    if (int rc = fsl_batch_step(b, 1)) return rc;
    return fsl_batch_get_positions_packed(b, out);
  }
  const size_t bytes = sizeof(double) * (size_t)b->packed_n;
  fsl::Exec& e = b->exec;
  e.io_in = [b, in, bytes](cudaStream_t st) {
    if (bytes) cudaMemcpyAsync(b->d_packed, in, bytes, cudaMemcpyHostToDevice, st);
    pack_on(b, 1, st);
  };
  e.io_out = [b, out, bytes](cudaStream_t st) {
    pack_on(b, 0, st);
    if (bytes) cudaMemcpyAsync(out, b->d_packed, bytes, cudaMemcpyDeviceToHost, st);
  };
  e.io_key[0] = in;
  e.io_key[1] = out;
  const int rc = fsl::exec_step(e, 1);
  e.io_in = nullptr;
  e.io_out = nullptr;
  e.io_key[0] = e.io_key[1] = nullptr;
  if (rc) return rc;
  FSL_TRY(cudaStreamSynchronize(e.stream));
  return FSL_OK;
}

int fsl_batch_get_positions_packed(fsl_batch* b, double* out) {
  int rc = fsl_batch_get_positions_packed_async(b, out);
  if (rc) return rc;
  FSL_TRY(cudaStreamSynchronize(b->exec.stream));
  return FSL_OK;
}

int fsl_batch_set_positions_packed(fsl_batch* b, const double* in) {
  int rc = fsl_batch_set_positions_packed_async(b, in);
  if (rc) return rc;
  FSL_TRY(cudaStreamSynchronize(b->exec.stream));
  return FSL_OK;
}

int fsl_batch_set_graph(fsl_batch* b, int enable) {
  if (!b) return errorf(FSL_E_ARG, "null batch");
  b->exec.use_graph = enable != 0;
  return FSL_OK;
}

int fsl_batch_get_info(fsl_batch* b, fsl_batch_info* info) {
  if (!b || !info) return errorf(FSL_E_ARG, "null argument");
  std::memset(info, 0, sizeof(*info));
  info->n = (int32_t)b->slots.size();
  info->classes = (int32_t)b->groups.size();
  info->graph = b->exec.gexec != nullptr;
  info->launches_per_step = b->exec.launches_per_step;
  info->np_total = b->packed_n / 3;
  info->nc_total = b->nc_total;
  int64_t bytes = 0;
  for (const auto& s : b->slots) bytes += (int64_t)s->bytes;
  bytes += (int64_t)sizeof(double) * b->packed_n;
  info->device_bytes = bytes;
  return FSL_OK;
}

int fsl_batch_get_class_tuning(fsl_batch* b, int32_t k, fsl_class_tuning* out) {
  if (!b || !out) return errorf(FSL_E_ARG, "null argument");
  if (k < 0 || k >= (int32_t)b->groups.size()) return errorf(FSL_E_ARG, "no size class %d", (int)k);
  auto it = b->groups.begin();
  std::advance(it, k);
  fsl::group_tuning(*it->second, out);
  return FSL_OK;
}

}  // extern "C"
