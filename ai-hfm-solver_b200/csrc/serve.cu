// Continuous-batching server over multigrid handles (hfm_serve_*): the serving loop for
// hosts that are not Python.
//
// One bucket per cubic edge: a handle with `slots` slots on a stream of its own, a pinned
// buffer the per-slot statistics are copied into after each launch, and an event recorded
// after that copy.  hfm_serve_poll visits every bucket: when its last launch has completed
// (event query, never a wait) it retires the slots that have finished - the float64
// solution is copied to the request's output on the bucket's stream and the request is
// reported once that copy's event has completed - admits queued requests into the free
// slots (conductivity hierarchy and right-hand side loaded for that slot only) and launches
// the bucket again.  Buckets never wait for one another.
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "hfm_internal.cuh"

namespace {

struct Request {
  int64_t ticket;
  int n;
  const float *sx, *sy, *sz, *f;
  double *x;
  bool cancel;
};

struct Copy {
  cudaEvent_t ev;
  hfm_serve_result res;
};

struct Bucket {
  int n = 0, slots = 0;
  hfm_mg *mg = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  hfm_slot_stats *stats = nullptr;  // pinned host memory, one entry per slot
  std::vector<int> free;            // free slots (popped from the back)
  std::vector<std::unique_ptr<Request>> busy;  // per slot: the request it holds
  std::deque<std::unique_ptr<Request>> queue;
  bool inflight = false;
  std::vector<int> launched;        // slots busy at the last launch
  std::vector<Copy> copies;         // solutions on their way to the requests' outputs
  std::vector<cudaEvent_t> spare;   // recycled copy events
};

}  // namespace

struct hfm_server {
  hfm_serve_config cfg;
  std::vector<std::unique_ptr<Bucket>> buckets;
  std::map<int, Bucket *> by_edge;
  int64_t next_ticket = 0;
  std::vector<hfm_serve_result> ready;  // results to report without a device copy (cancelled)
};

using namespace hfm;

namespace {

int destroy_bucket(Bucket *b) {
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto &c : b->copies) cudaEventDestroy(c.ev);
  for (auto e : b->spare) cudaEventDestroy(e);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->mg) hfm_mg_destroy(b->mg);
  if (b->stats) cudaFreeHost(b->stats);
  if (b->stream) cudaStreamDestroy(b->stream);
  return HFM_OK;
}

hfm_serve_result result_of(const Request &r, const hfm_slot_stats &s, int status) {
  hfm_serve_result o;
  o.ticket = r.ticket;
  o.status = status;
  o.cycles = s.cycles;
  o.outer = s.outer;
  o.rel_resid = s.rel_resid;
  return o;
}

// Retire the finished slots of the bucket's completed launch.
int harvest(hfm_server *srv, Bucket *b) {
  b->inflight = false;
  for (int slot : b->launched) {
    std::unique_ptr<Request> &r = b->busy[slot];
    if (!r) continue;
    const hfm_slot_stats &s = b->stats[slot];
    if (s.active) continue;
    if (r->cancel) {
      srv->ready.push_back(result_of(*r, s, HFM_ERR_CANCELLED));
    } else {
      int st = hfm_mg_fetch_f64(b->mg, slot, r->x, (hfm_stream_t)b->stream);
      if (st) return st;
      Copy c;
      if (!b->spare.empty()) {
        c.ev = b->spare.back();
        b->spare.pop_back();
      } else {
        HFM_CUDA(cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming));
      }
      HFM_CUDA(cudaEventRecord(c.ev, b->stream));
      c.res = result_of(*r, s, s.status);
      b->copies.push_back(c);
    }
    r.reset();
    b->free.push_back(slot);
  }
  return HFM_OK;
}

// Load a queued request into a free slot of its bucket (on the bucket's stream).
int admit(Bucket *b, std::unique_ptr<Request> req) {
  const int slot = b->free.back();
  b->free.pop_back();
  hfm_operator op;
  memset(&op, 0, sizeof(op));
  op.kind = HFM_OP_SIGMA7;
  op.coef_dtype = HFM_F32;
  op.scale = 1.f;
  op.c[0] = op.c[1] = op.c[2] = 1.f;
  op.coef[0] = req->sx;
  op.coef[1] = req->sy;
  op.coef[2] = req->sz;
  int st = hfm_mg_set_operator(b->mg, slot, &op, (hfm_stream_t)b->stream);
  if (!st) st = hfm_mg_load(b->mg, slot, req->f, nullptr, (hfm_stream_t)b->stream);
  b->busy[slot] = std::move(req);
  return st;
}

}  // namespace

extern "C" {

void hfm_serve_config_default(hfm_serve_config *c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  const int edges[5] = {32, 48, 64, 96, 128};
  c->n_edges = 5;
  for (int i = 0; i < 5; ++i) c->edges[i] = edges[i];
  c->slots = 64;
  c->budget_bytes = 120e9;
  c->cycles_per_tick = 4;
  hfm_mg_config_default(&c->solver);
  c->solver.op_kind = HFM_OP_SIGMA7;
  c->solver.cycle = HFM_CYCLE_V;
  c->solver.accel = HFM_ACCEL_IR;
  c->solver.storage = HFM_BF16;
  c->solver.tol = 1e-6;
  c->solver.inner_tol = 1e-3;
  c->solver.max_cycles = 600;
}

int hfm_serve_create(const hfm_serve_config *cfg, hfm_server **out) {
  if (!cfg || !out) return fail(HFM_ERR_BAD_ARG, "hfm_serve_create: NULL argument");
  *out = nullptr;
  const hfm_serve_config &c = *cfg;
  if (c.n_edges < 1 || c.n_edges > HFM_SERVE_MAX_EDGES)
    return fail(HFM_ERR_BAD_ARG, "hfm_serve_create: 1 .. 16 edges");
  if (c.slots < 1 || c.slots > 65535 || c.cycles_per_tick < 1 || !(c.budget_bytes > 0))
    return fail(HFM_ERR_BAD_ARG, "hfm_serve_create: bad slots / cycles_per_tick / budget");
  if (c.solver.op_kind != HFM_OP_SIGMA7 || c.solver.accel != HFM_ACCEL_IR)
    return fail(HFM_ERR_UNSUPPORTED, "hfm_serve_create: buckets solve SIGMA7 with float64 refinement (accel IR)");
  for (int i = 0; i < c.n_edges; ++i) {
    if (c.edges[i] < 2) return fail(HFM_ERR_BAD_ARG, "hfm_serve_create: edge < 2");
    for (int j = 0; j < i; ++j)
      if (c.edges[j] == c.edges[i]) return fail(HFM_ERR_BAD_ARG, "hfm_serve_create: repeated edge");
  }
  // admission by footprint: halve the largest bucket until every bucket fits the budget
  std::vector<double> per(c.n_edges);
  std::vector<int> want(c.n_edges, c.slots);
  for (int i = 0; i < c.n_edges; ++i)
    per[i] = (double)hfm_mg_footprint_bytes(&c.solver, c.edges[i], c.edges[i], c.edges[i], 1);
  for (;;) {
    double tot = 0;
    int big = 0;
    for (int i = 0; i < c.n_edges; ++i) {
      tot += per[i] * want[i];
      if (per[i] * want[i] > per[big] * want[big]) big = i;
    }
    if (tot <= c.budget_bytes) break;
    if (want[big] <= 1) return fail(HFM_ERR_OOM, "hfm_serve_create: the HBM budget holds less than one slot per edge");
    want[big] = std::max(1, want[big] / 2);
  }
  std::unique_ptr<hfm_server> srv(new hfm_server());
  srv->cfg = c;
  int st = HFM_OK;
  for (int i = 0; i < c.n_edges && !st; ++i) {
    std::unique_ptr<Bucket> b(new Bucket());
    b->n = c.edges[i];
    b->slots = want[i];
    st = hfm_mg_create(&c.solver, b->n, b->n, b->n, b->slots, &b->mg);
    if (!st && cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
      st = fail(HFM_ERR_CUDA, "hfm_serve_create: cudaStreamCreate failed");
    if (!st && cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess)
      st = fail(HFM_ERR_CUDA, "hfm_serve_create: cudaEventCreate failed");
    if (!st && cudaHostAlloc((void **)&b->stats, sizeof(hfm_slot_stats) * b->slots, cudaHostAllocDefault) != cudaSuccess)
      st = fail(HFM_ERR_OOM, "hfm_serve_create: pinned statistics buffer");
    if (!st) {
      b->busy.resize(b->slots);
      for (int s = b->slots - 1; s >= 0; --s) b->free.push_back(s);
      srv->by_edge[b->n] = b.get();
    }
    srv->buckets.push_back(std::move(b));
  }
  if (st) {
    for (auto &b : srv->buckets) destroy_bucket(b.get());
    return st;
  }
  *out = srv.release();
  return HFM_OK;
}

int hfm_serve_bucket_slots(const hfm_server *srv, int edge, int *slots) {
  if (!srv || !slots) return fail(HFM_ERR_BAD_ARG, "hfm_serve_bucket_slots: NULL argument");
  auto it = srv->by_edge.find(edge);
  if (it == srv->by_edge.end()) return fail(HFM_ERR_BAD_ARG, "hfm_serve_bucket_slots: edge not served");
  *slots = it->second->slots;
  return HFM_OK;
}

int hfm_serve_submit(hfm_server *srv, int n, const float *sx, const float *sy, const float *sz,
                     const float *f, double *x, int64_t *ticket) {
  if (!srv || !sx || !sy || !sz || !f || !x || !ticket)
    return fail(HFM_ERR_BAD_ARG, "hfm_serve_submit: NULL argument");
  auto it = srv->by_edge.find(n);
  if (it == srv->by_edge.end()) return fail(HFM_ERR_BAD_ARG, "hfm_serve_submit: edge not served");
  std::unique_ptr<Request> r(new Request{srv->next_ticket++, n, sx, sy, sz, f, x, false});
  *ticket = r->ticket;
  it->second->queue.push_back(std::move(r));
  return HFM_OK;
}

int hfm_serve_poll(hfm_server *srv, hfm_serve_result *done, int cap, int *n_done) {
  if (!srv || !n_done || cap < 0 || (cap > 0 && !done)) return fail(HFM_ERR_BAD_ARG, "hfm_serve_poll: bad argument");
  *n_done = 0;
  int st;
  for (auto &bp : srv->buckets) {
    Bucket *b = bp.get();
    // solutions whose copy has completed
    for (size_t i = 0; i < b->copies.size();) {
      cudaError_t e = cudaEventQuery(b->copies[i].ev);
      if (e == cudaErrorNotReady) {
        ++i;
        continue;
      }
      if (e != cudaSuccess) return cuda_status(e, "hfm_serve_poll: cudaEventQuery");
      srv->ready.push_back(b->copies[i].res);
      b->spare.push_back(b->copies[i].ev);
      b->copies.erase(b->copies.begin() + i);
    }
    if (b->inflight) {
      cudaError_t e = cudaEventQuery(b->ev);
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess) return cuda_status(e, "hfm_serve_poll: cudaEventQuery");
      if ((st = harvest(srv, b))) return st;
    }
    // cancelled requests still in a slot: stop them (stream-ordered before any reuse)
    for (int slot = 0; slot < b->slots; ++slot)
      if (b->busy[slot] && b->busy[slot]->cancel) {
        if ((st = hfm_mg_cancel(b->mg, slot, (hfm_stream_t)b->stream))) return st;
        hfm_slot_stats zero;
        memset(&zero, 0, sizeof(zero));
        srv->ready.push_back(result_of(*b->busy[slot], zero, HFM_ERR_CANCELLED));
        b->busy[slot].reset();
        b->free.push_back(slot);
      }
    while (!b->queue.empty() && !b->free.empty()) {
      std::unique_ptr<Request> r = std::move(b->queue.front());
      b->queue.pop_front();
      if ((st = admit(b, std::move(r)))) return st;
    }
    b->launched.clear();
    for (int slot = 0; slot < b->slots; ++slot)
      if (b->busy[slot]) b->launched.push_back(slot);
    if (b->launched.empty()) continue;
    if ((st = hfm_mg_run(b->mg, srv->cfg.cycles_per_tick, (hfm_stream_t)b->stream))) return st;
    if ((st = hfm_mg_query_async(b->mg, b->stats, (hfm_stream_t)b->stream))) return st;
    HFM_CUDA(cudaEventRecord(b->ev, b->stream));
    b->inflight = true;
  }
  int k = 0;
  while (k < cap && !srv->ready.empty()) {
    done[k++] = srv->ready.front();
    srv->ready.erase(srv->ready.begin());
  }
  *n_done = k;
  return HFM_OK;
}

int hfm_serve_cancel(hfm_server *srv, int64_t ticket) {
  if (!srv) return fail(HFM_ERR_BAD_ARG, "hfm_serve_cancel: NULL server");
  for (auto &bp : srv->buckets) {
    Bucket *b = bp.get();
    for (auto it = b->queue.begin(); it != b->queue.end(); ++it)
      if ((*it)->ticket == ticket) {
        hfm_slot_stats zero;
        memset(&zero, 0, sizeof(zero));
        srv->ready.push_back(result_of(**it, zero, HFM_ERR_CANCELLED));
        b->queue.erase(it);
        return HFM_OK;
      }
    for (auto &r : b->busy)
      if (r && r->ticket == ticket) {
        if (r->cancel) break;
        r->cancel = true;  // stopped at the bucket's next visit by hfm_serve_poll
        return HFM_OK;
      }
  }
  return fail(HFM_ERR_BAD_ARG, "hfm_serve_cancel: unknown, finished or already cancelled ticket");
}

int hfm_serve_pending(const hfm_server *srv, int *queued, int *running) {
  if (!srv || !queued || !running) return fail(HFM_ERR_BAD_ARG, "hfm_serve_pending: NULL argument");
  int q = 0, r = 0;
  for (auto &bp : srv->buckets) {
    q += (int)bp->queue.size();
    for (auto &x : bp->busy) r += x ? 1 : 0;
    r += (int)bp->copies.size();
  }
  *queued = q;
  *running = r;
  return HFM_OK;
}

int hfm_serve_destroy(hfm_server *srv) {
  if (!srv) return HFM_OK;
  for (auto &b : srv->buckets) destroy_bucket(b.get());
  delete srv;
  return HFM_OK;
}

}  // extern "C"
