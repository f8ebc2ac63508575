// dim2d_server.cu -- serving loop (include/dim2d.h, dim2d_server_*).  No
// counterpart in the reference (one solve per process there).
//
// Requests (a field's initial state, dt, step count) arrive at any time
// through dim2d_server_submit.  dim2d_server_poll drives the loop:
//   1. retire: requests whose result copy has landed are complete; their
//      fields are destroyed and their memory returns to the budget;
//   2. admit: pending requests, in arrival order, while their three device
//      copies fit the memory budget -- each becomes a field (created,
//      uploaded, node boundary pass) and joins the running batch;
//   3. run: while fewer than two chunks are in flight, enqueue the next
//      chunk of min(chunk_steps, smallest remaining step count) batched
//      steps; requests that reach their step count get their result copied
//      to host memory right behind that chunk (same stream) and leave the
//      batch before the next chunk is built.
//   4. check: behind every chunk, one small kernel per member sets the
//      member's health word if its state holds a non-finite value or its
//      wall root failed (where the reference stops); the word travels to
//      pinned host memory behind the chunk, and a flagged request leaves
//      the batch at the next chunk boundary with the state it has, instead
//      of being stepped to its last step.
// So requests that arrive while others run are admitted as memory frees
// up and advance in the same batched launches (continuous batching), and
// the GPU always has the next chunk queued while the host admits/retires.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "dim2d_internal.h"

using namespace dim2d;

namespace {
using Clock = std::chrono::steady_clock;

enum ReqState : int { R_PENDING = 0, R_ACTIVE, R_COPYING, R_DONE };

struct Request {
  long long id = 0;
  int nx = 0, ny = 0, precision = 0;
  int bc_choice[8]{}, bc_type[8]{}, bc_order[8]{};
  double* staging = nullptr;  // pinned: nodes (4 nx ny), x_map (nx), y_map (ny)
  size_t staging_cap = 0;
  double dt = 0;
  long long nsteps = 0, remaining = 0;
  size_t bytes = 0;
  ReqState state = R_PENDING;
  dim2d_handle* h = nullptr;
  double* result = nullptr;  // pinned: final state (4 nx ny) + wall status word
  size_t result_cap = 0;
  unsigned int status = 0;
  unsigned int stopped = 0;  // health flags of a request that left early (or finished flagged)
  double t_final = 0;
  cudaEvent_t copied = nullptr;
  Clock::time_point t_submit, t_done;
};

struct Chunk {
  cudaEvent_t done = nullptr;
};
}  // namespace

struct dim2d_server {
  dim2d_params p{};
  int device = 0;
  size_t budget = 0, used = 0;
  int chunk_steps = 500;
  dim2d_batch* batch = nullptr;
  cudaStream_t stream = nullptr;
  long long next_id = 1;
  std::deque<Request*> pending;
  std::vector<Request*> active;   // members of the batch
  std::vector<Request*> copying;  // result copy in flight
  std::map<long long, Request*> all;
  std::deque<Chunk> inflight;
  std::vector<cudaEvent_t> free_events;
  std::multimap<size_t, double*> pinned_free;  // reusable pinned buffers by capacity
  std::vector<double*> pinned_all;
  long long completed = 0, cell_updates = 0;
  int max_active = 0;
};

namespace {

// health word of a field: bit 0 if any value of its interior cells (4
// planes) is not finite, bit 1 if its wall root status word is set.  Words
// are only ever set (the conditions are terminal), so no reset is needed
// between chunks.  (A ghost cell that blows up reaches the interior within
// a step or two; the ghost cells of some presets are not all defined.)
__global__ void k_health(const double* __restrict__ u, Field f, const unsigned int* status,
                         unsigned int* out) {
  bool bad = false;
  const size_t nxi = (size_t)(f.nx - 2 * BC);
  const size_t per_plane = (size_t)(f.ny - 2 * BC) * nxi;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < 4 * per_plane;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t v = i / per_plane, r = i % per_plane;
    const size_t y = BC + r / nxi, x = BC + r % nxi;
    bad |= !isfinite(u[v * f.plane + y * f.pitch + x]);
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    unsigned int w = bad ? 1u : 0u;
    if (blockIdx.x == 0 && status && *status) w |= 2u;
    if (w) atomicOr(out, w);
  }
}

cudaError_t launch_health(dim2d_handle* h, cudaStream_t s) {
  const size_t n = 4 * (size_t)(h->f.ny - 2 * BC) * (h->f.nx - 2 * BC);
  // grid-stride: at most 4 CTAs of 256 threads per SM on a 148-SM B200
  const unsigned blocks = (unsigned)std::min<size_t>(592, (n + 255) / 256);
  k_health<<<blocks, 256, 0, s>>>(h->A, h->f, h->south_wall ? h->status : nullptr,
                                  health_word(h));
  return cudaGetLastError();
}

// pinned host copy of a request's health word: the slot after the status
// word behind the result state
unsigned int* health_host(Request* r) {
  return reinterpret_cast<unsigned int*>(r->result + 4 * (size_t)r->nx * r->ny + 1);
}

cudaEvent_t get_event(dim2d_server* s) {
  if (!s->free_events.empty()) {
    cudaEvent_t e = s->free_events.back();
    s->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  return e;
}

// Pinned host buffers are kept and reused: allocating and freeing pinned
// memory is slow and freeing it synchronises the device.
double* pinned_get(dim2d_server* s, size_t n, size_t* cap) {
  auto it = s->pinned_free.lower_bound(n);
  if (it != s->pinned_free.end() && it->first <= 2 * n) {
    double* p = it->second;
    *cap = it->first;
    s->pinned_free.erase(it);
    return p;
  }
  size_t c = 1024;
  while (c < n) c *= 2;
  double* p = nullptr;
  if (cudaMallocHost((void**)&p, c * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  s->pinned_all.push_back(p);
  *cap = c;
  return p;
}

void pinned_put(dim2d_server* s, double* p, size_t cap) {
  if (p) s->pinned_free.emplace(cap, p);
}

size_t request_bytes(int nx, int ny) {
  // three pitched FP64 copies of 4 planes plus x_map/y_map and slack
  return 3 * 4 * (size_t)ny * (size_t)pitch_for(nx) * sizeof(double) + 2 * 4096 +
         (size_t)(nx + ny) * sizeof(double);
}

void release(dim2d_server* s, Request* r) {
  if (r->h) {
    dim2d_destroy(r->h);
    r->h = nullptr;
    s->used -= r->bytes;
  }
}

int retire(dim2d_server* s, int* completed) {
  // chunks that have finished
  while (!s->inflight.empty() && cudaEventQuery(s->inflight.front().done) == cudaSuccess) {
    s->free_events.push_back(s->inflight.front().done);
    s->inflight.pop_front();
  }
  cudaGetLastError();  // cudaErrorNotReady from the queries
  for (size_t i = 0; i < s->copying.size();) {
    Request* r = s->copying[i];
    const cudaError_t e = cudaEventQuery(r->copied);
    if (e == cudaErrorNotReady) {
      cudaGetLastError();
      i++;
      continue;
    }
    if (e != cudaSuccess) return cuda_error(e, "server retire");
    r->t_done = Clock::now();
    r->state = R_DONE;
    std::memcpy(&r->status, r->result + 4 * (size_t)r->nx * r->ny, sizeof r->status);
    r->stopped |= *health_host(r);
    s->free_events.push_back(r->copied);
    r->copied = nullptr;
    release(s, r);
    pinned_put(s, r->staging, r->staging_cap);
    r->staging = nullptr;
    s->copying.erase(s->copying.begin() + i);
    s->completed++;
    if (completed) (*completed)++;
  }
  return DIM2D_OK;
}

int admit(dim2d_server* s) {
  while (!s->pending.empty()) {
    Request* r = s->pending.front();
    if (s->used + r->bytes > s->budget) break;  // admission by free memory
    dim2d_handle* h = nullptr;
    // buffers from the stream-ordered pool on the server's stream
    int rc = create_field(&s->p, r->nx, r->ny, r->bc_choice, r->bc_type, r->bc_order,
                          r->precision, s->stream, &h);
    const size_t n = 4 * (size_t)r->nx * r->ny;
    if (!rc) rc = dim2d_upload(h, r->staging, r->staging + n, r->staging + n + r->nx, 0.0);
    if (!rc && !h->periodic && !h->open_all) rc = dim2d_apply_bc_on_nodes(h);  // field%ini
    if (!rc) rc = dim2d_batch_add(s->batch, h, r->dt);
    if (rc) {
      if (h) dim2d_destroy(h);
      return rc;
    }
    r->h = h;
    s->used += r->bytes;
    r->state = R_ACTIVE;
    s->pending.pop_front();
    s->active.push_back(r);
  }
  s->max_active = std::max(s->max_active, (int)s->active.size());
  return DIM2D_OK;
}

// final state -> pinned host memory, right behind the work queued so far;
// the request leaves the batch
int finish(dim2d_server* s, Request* r) {
  const Field& f = r->h->f;
  cudaError_t e = cudaMemcpy2DAsync(r->result, f.nx * sizeof(double), r->h->A, f.pitch * sizeof(double),
                                    f.nx * sizeof(double), 4 * (size_t)f.ny,
                                    cudaMemcpyDeviceToHost, s->stream);
  unsigned int* st = reinterpret_cast<unsigned int*>(r->result + 4 * (size_t)f.nx * f.ny);
  *st = 0;
  if (e == cudaSuccess && r->h->south_wall)  // wall root status word, behind the state
    e = cudaMemcpyAsync(st, r->h->status, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                        s->stream);
  r->copied = get_event(s);
  if (e == cudaSuccess) e = cudaEventRecord(r->copied, s->stream);
  if (e != cudaSuccess) return cuda_error(e, "server result copy");
  r->t_final = r->h->t;
  const int rc = dim2d_batch_remove(s->batch, r->h);
  if (rc) return rc;
  r->state = R_COPYING;
  s->copying.push_back(r);
  return DIM2D_OK;
}

int run_chunk(dim2d_server* s) {
  // requests an earlier chunk's check flagged leave now, with the state
  // they have (the words read here may be a chunk old: flags only get set)
  for (size_t i = 0; i < s->active.size();) {
    Request* r = s->active[i];
    const unsigned int flags = *(volatile unsigned int*)health_host(r);
    if (!flags) {
      i++;
      continue;
    }
    r->stopped = flags;
    const int rc = finish(s, r);
    if (rc) return rc;
    s->active.erase(s->active.begin() + i);
  }
  if (s->active.empty()) return DIM2D_OK;
  long long k = s->chunk_steps;
  for (Request* r : s->active) k = std::min(k, r->remaining);
  int rc = dim2d_batch_step(s->batch, (int)k);
  if (rc) return rc;
  // health checks of every member behind the chunk, their words to the host
  cudaError_t e = cudaSuccess;
  for (Request* r : s->active) {
    e = launch_health(r->h, s->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(health_host(r), health_word(r->h), sizeof(unsigned int),
                          cudaMemcpyDeviceToHost, s->stream);
    if (e != cudaSuccess) return cuda_error(e, "server health check");
  }
  Chunk c;
  c.done = get_event(s);
  e = cudaEventRecord(c.done, s->stream);
  if (e != cudaSuccess) return cuda_error(e, "server chunk");
  s->inflight.push_back(c);
  for (size_t i = 0; i < s->active.size();) {
    Request* r = s->active[i];
    r->remaining -= k;
    s->cell_updates += k * (long long)(r->nx - 2 * BC) * (r->ny - 2 * BC);
    if (r->remaining > 0) {
      i++;
      continue;
    }
    rc = finish(s, r);
    if (rc) return rc;
    s->active.erase(s->active.begin() + i);
  }
  return DIM2D_OK;
}

}  // namespace

extern "C" {

int dim2d_server_create(const dim2d_params* p, size_t mem_budget, int chunk_steps,
                        dim2d_server** out) {
  if (!p || !out || chunk_steps <= 0) return set_error(DIM2D_ERR_ARG, "server_create: bad argument");
  *out = nullptr;
  dim2d_server* s = new dim2d_server();
  s->p = *p;
  s->chunk_steps = chunk_steps;
  cudaGetDevice(&s->device);
  size_t free_b = 0, total_b = 0;
  cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) {
    delete s;
    return cuda_error(e, "server_create");
  }
  // default budget: the free memory less 10% (or 4 GiB, if smaller) of slack
  const size_t reserve = std::min<size_t>(free_b / 10, (size_t)4 << 30);
  s->budget = mem_budget ? std::min(mem_budget, free_b - reserve) : free_b - reserve;
  // keep memory released by retired fields in the device's stream-ordered
  // pool for the next admissions instead of returning it at every
  // synchronisation (a property of this process's pool, not of the GPU)
  cudaMemPool_t mp = nullptr;
  if (cudaDeviceGetDefaultMemPool(&mp, s->device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  int rc = dim2d_batch_create(&s->batch);
  if (rc) {
    delete s;
    return rc;
  }
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    dim2d_batch_destroy(s->batch);
    delete s;
    return cuda_error(e, "server_create");
  }
  dim2d_batch_set_stream(s->batch, s->stream);
  *out = s;
  return DIM2D_OK;
}

int dim2d_server_submit(dim2d_server* s, int nx, int ny, const int bc_choice[8],
                        const int bc_type[8], const int bc_order[8], int precision,
                        const double* nodes, const double* x_map, const double* y_map, double dt,
                        long long nsteps, long long* id) {
  if (!s || !bc_choice || !bc_type || !bc_order || !nodes || !x_map || !y_map || !id)
    return set_error(DIM2D_ERR_ARG, "server_submit: null argument");
  if (nx < 8 || ny < 8 || nsteps <= 0 || !(dt > 0) || !std::isfinite(dt))
    return set_error(DIM2D_ERR_ARG, "server_submit: bad size, dt or step count");
  if (precision != DIM2D_FP64 && precision != DIM2D_MIXED)
    return set_error(DIM2D_ERR_ARG, "server_submit: unknown precision %d", precision);
  Request* r = new Request();
  r->bytes = request_bytes(nx, ny);
  if (r->bytes > s->budget) {
    delete r;
    return set_error(DIM2D_ERR_NOMEM, "server_submit: a %dx%d field exceeds the memory budget",
                     nx, ny);
  }
  r->id = s->next_id++;
  r->nx = nx;
  r->ny = ny;
  r->precision = precision;
  std::memcpy(r->bc_choice, bc_choice, sizeof r->bc_choice);
  std::memcpy(r->bc_type, bc_type, sizeof r->bc_type);
  std::memcpy(r->bc_order, bc_order, sizeof r->bc_order);
  const size_t n = 4 * (size_t)nx * ny;
  r->staging = pinned_get(s, n + nx + ny, &r->staging_cap);
  r->result = pinned_get(s, n + 2, &r->result_cap);
  if (!r->staging || !r->result) {
    pinned_put(s, r->staging, r->staging_cap);
    pinned_put(s, r->result, r->result_cap);
    delete r;
    return set_error(DIM2D_ERR_NOMEM, "server_submit: pinned host buffers");
  }
  *health_host(r) = 0;
  std::memcpy(r->staging, nodes, n * sizeof(double));
  std::memcpy(r->staging + n, x_map, nx * sizeof(double));
  std::memcpy(r->staging + n + nx, y_map, ny * sizeof(double));
  r->dt = dt;
  r->nsteps = r->remaining = nsteps;
  r->t_submit = Clock::now();
  s->pending.push_back(r);
  s->all[r->id] = r;
  *id = r->id;
  return DIM2D_OK;
}

int dim2d_server_poll(dim2d_server* s, int wait, int* completed) {
  if (!s) return set_error(DIM2D_ERR_ARG, "server_poll: null server");
  if (completed) *completed = 0;
  if (wait && !s->inflight.empty()) {
    cudaError_t e = cudaEventSynchronize(s->inflight.front().done);
    if (e != cudaSuccess) return cuda_error(e, "server_poll");
  }
  int rc = retire(s, completed);
  if (!rc) rc = admit(s);
  while (!rc && s->inflight.size() < 2 && !s->active.empty()) rc = run_chunk(s);
  if (!rc && wait && s->active.empty() && !s->copying.empty()) {
    // nothing left to run: wait for the last result copies
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_error(e, "server_poll");
    rc = retire(s, completed);
  }
  return rc;
}

int dim2d_server_result(dim2d_server* s, long long id, double* nodes, double* t,
                        double* latency_s) {
  if (!s) return set_error(DIM2D_ERR_ARG, "server_result: null server");
  auto it = s->all.find(id);
  if (it == s->all.end()) return set_error(DIM2D_ERR_ARG, "server_result: unknown request %lld", id);
  Request* r = it->second;
  if (r->state != R_DONE) return DIM2D_ERR_NOT_READY;
  if (nodes) std::memcpy(nodes, r->result, 4 * (size_t)r->nx * r->ny * sizeof(double));
  if (t) *t = r->t_final;
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  const unsigned int status = r->status, stopped = r->stopped;
  const long long done = r->nsteps - r->remaining;
  pinned_put(s, r->result, r->result_cap);
  s->all.erase(it);
  delete r;
  if (status)  // the reference stops where a wall ghost root fails
    return set_error(DIM2D_ERR_WALL_ROOT, "request %lld: wall ghost cell root (status 0x%x)",
                     id, status);
  if (stopped & 1u)
    return set_error(DIM2D_ERR_NONFINITE,
                     "request %lld: state not finite (stopped after %lld steps)", id, done);
  return DIM2D_OK;
}

int dim2d_server_stats(const dim2d_server* s, long long out[8]) {
  if (!s || !out) return set_error(DIM2D_ERR_ARG, "server_stats: null argument");
  out[0] = (long long)s->pending.size();
  out[1] = (long long)s->active.size();
  out[2] = (long long)s->copying.size();
  out[3] = s->completed;
  out[4] = s->cell_updates;
  out[5] = (long long)s->used;
  out[6] = (long long)s->budget;
  out[7] = s->max_active;
  return DIM2D_OK;
}

int dim2d_server_destroy(dim2d_server* s) {
  if (!s) return DIM2D_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto& kv : s->all) {
    Request* r = kv.second;
    if (r->h && s->batch) dim2d_batch_remove(s->batch, r->h);
    release(s, r);
    if (r->copied) cudaEventDestroy(r->copied);
    delete r;
  }
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (double* p : s->pinned_all) cudaFreeHost(p);
  for (Chunk& c : s->inflight) cudaEventDestroy(c.done);
  for (cudaEvent_t e : s->free_events) cudaEventDestroy(e);
  if (s->batch) dim2d_batch_destroy(s->batch);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DIM2D_OK;
}

}  // extern "C"
