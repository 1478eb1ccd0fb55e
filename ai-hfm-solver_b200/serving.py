"""Continuous-batching server for anisotropic forward solves of mixed grid sizes.

Requests (sigma, f, arrival time) of different cubic edges arrive over time.  The server
keeps one resident multigrid handle per edge ("bucket") with a fixed number of slots whose
hierarchies live in HBM, sized so the buckets fit an HBM budget (admission by footprint,
``hfm_mg_footprint_bytes``).  The serving loop

1. admits every request that has arrived into a free slot of its bucket (coefficient
   hierarchy + right-hand side loaded into that slot; requests wait in a queue while their
   bucket is full);
2. advances every bucket that holds work by a few cycles (one CUDA-graph launch per bucket,
   each bucket on its own stream so the buckets overlap on the GPU); inside the graph every
   slot runs on its own: a slot that converges, fails or hits its cycle cap switches itself
   off and the remaining kernels skip it;
3. as soon as a bucket's own launch has completed (non-blocking event check on an
   asynchronous copy of the per-slot statistics), retires its finished slots (solution copied
   out, latency recorded), admits waiting requests into the freed slots and launches the
   bucket again; buckets of different sizes never wait for one another.

A request that arrives while others are on the GPU therefore joins the next launch of its
bucket: iteration-level continuous batching, not a queue that waits for a batch to drain.
Requests whose inputs are in host memory start their host -> device copy on arrival (copy
stream), so the copies of queued requests overlap the buckets' work.
Each slot's arithmetic depends only on its own data (fixed-order per-slot reductions), so a
result is the same alone and in the mix.

The plain baseline (``solve_one_at_a_time``) is the same solver with one slot per handle,
one request at a time, float32 storage.
"""
import collections
import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from .multigrid import Multigrid, SolverConfig, footprint_bytes
from .ops import Sigma7

EDGES = (32, 48, 64, 96, 128)


@dataclass
class SolveRequest:
    rid: int
    n: int
    arrival: float                 # seconds after the stream starts
    sigma: torch.Tensor            # (3, n, n, n) float32 (device, or pinned host for e2e)
    rhs: torch.Tensor              # (n, n, n) float32
    log_std: float = 1.0


@dataclass
class SolveResult:
    rid: int
    n: int
    status: int
    cycles: int
    outer: int
    rel_resid: float
    admitted: float
    done: float
    latency: float
    phi: torch.Tensor = None


def sigma_field(n, gen, log_std, device):
    """Seeded log-normal conductivity: iid N(0,1) per axis, 5^3 box filter with reflected
    edges, rescaled to mean 0 / std ``log_std``, exponentiated (same recipe as
    ``problems.anisotropic_sigma``, generated on the device)."""
    g = torch.randn((3, 1, n, n, n), device=device, generator=gen)
    g = torch.nn.functional.pad(g, (2, 2, 2, 2, 2, 2), mode="reflect")
    g = torch.nn.functional.avg_pool3d(g, 5, stride=1)[:, 0]
    m = g.mean(dim=(1, 2, 3), keepdim=True)
    s = g.std(dim=(1, 2, 3), keepdim=True)
    return torch.exp((g - m) / (s + 1e-30) * log_std).contiguous()


def dipole_field(n, rng, device, margin=4):
    f = torch.zeros((n, n, n), device=device)
    lo, hi = margin, n - margin
    p = tuple(int(v) for v in rng.integers(lo, hi, 3))
    q = p
    while q == p:
        q = tuple(int(v) for v in rng.integers(lo, hi, 3))
    f[p] = 1.0
    f[q] = -1.0
    return f


def make_stream(count=1024, rate=2000.0, edges=EDGES, log_std=(0.5, 2.0), seed=0,
                device="cuda", only=None):
    """The serving workload: ``count`` requests, edge uniform over ``edges``, log-std uniform
    in ``log_std``, own sigma and dipole each, Poisson arrivals at ``rate`` per second.
    With ``only`` (a set of request ids) the fields are built for those requests alone; the
    others keep their edge, arrival and log-std with ``sigma = rhs = None`` (the draws, and
    so every request, are the same either way)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    t = 0.0
    reqs = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice(edges))
        ls = float(rng.uniform(*log_std))
        if only is not None and i not in only:
            _dipole_draws(n, rng)
            reqs.append(SolveRequest(i, n, t, None, None, ls))
            continue
        gen.manual_seed(seed * 1000003 + i)
        reqs.append(SolveRequest(i, n, t, sigma_field(n, gen, ls, device),
                                 dipole_field(n, rng, device), ls))
    return reqs


def _dipole_draws(n, rng, margin=4):
    """The random draws of ``dipole_field`` without building the field."""
    lo, hi = margin, n - margin
    p = tuple(int(v) for v in rng.integers(lo, hi, 3))
    q = p
    while q == p:
        q = tuple(int(v) for v in rng.integers(lo, hi, 3))


def with_rate(requests, rate, seed=0):
    """The same requests with Poisson arrivals re-drawn at ``rate`` per second (order kept):
    the stream at a lower offered load."""
    rng = np.random.default_rng(seed + 7)
    t = 0.0
    out = []
    for r in requests:
        t += rng.exponential(1.0 / rate)
        out.append(SolveRequest(r.rid, r.n, t, r.sigma, r.rhs, r.log_std))
    return out


class _Bucket:
    """One edge size: a resident handle with ``slots`` slots on its own CUDA stream.  Launches
    are asynchronous: after each graph launch the per-slot statistics are copied into pinned
    host memory and an event is recorded; the server harvests the bucket when the event has
    completed, so buckets of different sizes never wait for one another."""

    def __init__(self, n, cfg, slots, keep_solutions):
        self.n = n
        self.slots = slots
        self.mg = Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=slots)
        self.stream = torch.cuda.Stream()
        self.free = list(range(slots - 1, -1, -1))
        self.busy = {}  # slot -> (request, admitted time, staging tensors)
        self.keep = keep_solutions
        self.stats_buf = torch.empty(slots * C.sizeof(L.HfmSlotStats), dtype=torch.uint8,
                                     pin_memory=True)
        self.event = torch.cuda.Event()
        self.inflight = False
        self.launched = ()
        self.copies = []  # solutions on their way to host memory: (event, result, host, dev)

    def ready(self):
        return not self.inflight or self.event.query()

    def admit(self, req, now, staged=None):
        """Load ``req`` into a free slot.  ``staged`` = (sigma, rhs, event): its inputs were
        already copied to the device on the server's copy stream (end-to-end mode)."""
        slot = self.free.pop()
        with torch.cuda.stream(self.stream):
            sig, rhs = req.sigma, req.rhs
            if staged is not None:
                sig, rhs, ev = staged
                self.stream.wait_event(ev)
                sig.record_stream(self.stream)
                rhs.record_stream(self.stream)
            elif not sig.is_cuda:  # host inputs not staged yet: copy them now
                sig = sig.to("cuda", non_blocking=True)
                rhs = rhs.to("cuda", non_blocking=True)
            self.mg.set_operator(Sigma7(sig[0], sig[1], sig[2]), slot=slot)
            self.mg.load(slot, rhs)
        # the staging tensors stay referenced until the slot retires
        self.busy[slot] = (req, now, (sig, rhs))

    def launch(self, cycles):
        if not self.busy:
            return
        with torch.cuda.stream(self.stream):
            self.mg.run(cycles)
            self.mg.query_async(self.stats_buf)
            self.event.record(self.stream)
        self.inflight = True
        self.launched = tuple(self.busy.keys())

    def harvest(self, clock, t0, host_out):
        """Retire the slots of the completed launch that have finished (call when ready()).
        With ``host_out`` a finished solution is copied into pinned host memory
        asynchronously on the bucket's stream; its result is reported by ``poll_copies``
        once that copy has completed, and the slot is free for the next request at once
        (later work on the slot is ordered after the copy by the stream)."""
        if not self.inflight:
            return []
        self.inflight = False
        stats = self.mg.decode_stats(self.stats_buf)
        done = []
        now = clock() - t0
        for slot in self.launched:
            s = stats[slot]
            if s["active"]:
                continue
            req, adm, _ = self.busy.pop(slot)
            self.free.append(slot)
            phi = None
            if self.keep or host_out:
                with torch.cuda.stream(self.stream):
                    phi = self.mg.fetch_f64(slot) if self.mg.cfg.accel == "ir" else self.mg.fetch(slot)
                    if host_out:
                        host = torch.empty(phi.shape, dtype=phi.dtype, pin_memory=True)
                        host.copy_(phi, non_blocking=True)
                        ev = torch.cuda.Event()
                        ev.record(self.stream)
                        res = SolveResult(req.rid, req.n, s["status"], s["cycles"], s["outer"],
                                          s["rel_resid"], adm, 0.0, 0.0, host)
                        self.copies.append((ev, res, host, phi, req))
                        continue
            done.append(SolveResult(req.rid, req.n, s["status"], s["cycles"], s["outer"],
                                    s["rel_resid"], adm, now, now - req.arrival, phi))
        return done

    def poll_copies(self, clock, t0):
        """Results whose solution has arrived in host memory (non-blocking)."""
        out, keep = [], []
        for item in self.copies:
            ev, res, _, _, req = item
            if ev.query():
                now = clock() - t0
                res.done, res.latency = now, now - req.arrival
                out.append(res)
            else:
                keep.append(item)
        self.copies = keep
        return out


class SolveServer:
    """Buckets per edge sized to an HBM budget; ``serve`` runs a request stream."""

    def __init__(self, cfg=None, edges=EDGES, slots=64, budget_bytes=120e9,
                 cycles_per_tick=4, keep_solutions=False):
        self.cfg = cfg or SolverConfig(cycle="V", accel="ir", storage="bf16", tol=1e-6,
                                       max_cycles=600, inner_tol=1e-3)
        self.cycles_per_tick = cycles_per_tick
        per = {n: footprint_bytes(self.cfg, L.OP_SIGMA7, (n, n, n), 1) for n in edges}
        want = {n: (slots[n] if isinstance(slots, dict) else slots) for n in edges}
        # admission by footprint: shrink the largest buckets until everything fits the budget
        while sum(per[n] * want[n] for n in edges) > budget_bytes:
            big = max(edges, key=lambda n: per[n] * want[n])
            if want[big] <= 1:
                raise ValueError("HBM budget too small for one slot per edge")
            want[big] = max(1, want[big] // 2)
        self.footprint = {n: per[n] * want[n] for n in edges}
        self.buckets = {n: _Bucket(n, self.cfg, want[n], keep_solutions) for n in edges}
        self.copy_stream = torch.cuda.Stream()

    def close(self):
        for b in self.buckets.values():
            b.mg.close()

    def serve(self, requests, realtime=True, host_out=False):
        """Serve ``requests`` (sorted by arrival).  With ``realtime`` a request is admitted only
        once its arrival time has passed on the wall clock.  Returns the list of results."""
        clock = time.perf_counter
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queued = {n: collections.deque() for n in self.buckets}
        staged = {}  # rid -> device copies of host inputs (end-to-end mode)
        results = []
        torch.cuda.synchronize()
        t0 = clock()
        total = len(pending)
        buckets = list(self.buckets.values())
        while len(results) < total:
            now = clock() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                r = pending.popleft()
                queued[r.n].append(r)
                if not r.sigma.is_cuda:
                    # host inputs start their copy to the device on arrival, on a stream of their
                    # own, so admission into a slot later does not wait for it
                    with torch.cuda.stream(self.copy_stream):
                        sd = r.sigma.to("cuda", non_blocking=True)
                        rd = r.rhs.to("cuda", non_blocking=True)
                        ev = torch.cuda.Event()
                        ev.record(self.copy_stream)
                    staged[r.rid] = (sd, rd, ev)
            idle = True
            for b in buckets:
                if b.copies:
                    results.extend(b.poll_copies(clock, t0))
                    idle = False
                if not b.ready():
                    idle = False
                    continue
                results.extend(b.harvest(clock, t0, host_out))
                q = queued[b.n]
                while q and b.free:
                    r = q.popleft()
                    b.admit(r, clock() - t0, staged.pop(r.rid, None))
                b.launch(self.cycles_per_tick)
                if b.inflight:
                    idle = False
            if idle and pending:
                wait = pending[0].arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(min(wait, 2e-4))
        torch.cuda.synchronize()
        return results


class NativeServer:
    """The library's own serving loop (``hfm_serve_*``, the C ABI a non-Python host calls):
    the same buckets, admission by footprint and per-bucket graph launches as
    ``SolveServer``, driven by ``hfm_serve_poll``."""

    def __init__(self, cfg=None, edges=EDGES, slots=64, budget_bytes=120e9, cycles_per_tick=4):
        c = L.HfmServeConfig()
        L.lib().hfm_serve_config_default(C.byref(c))
        c.n_edges = len(edges)
        for i, e in enumerate(edges):
            c.edges[i] = int(e)
        c.slots = int(slots)
        c.budget_bytes = float(budget_bytes)
        c.cycles_per_tick = int(cycles_per_tick)
        if cfg is not None:
            c.solver = cfg.struct(L.OP_SIGMA7)
        h = C.c_void_p()
        L.call("hfm_serve_create", C.byref(c), C.byref(h))
        self._h = h
        self._keep = {}  # ticket -> (inputs, output): valid until the request is reported

    def bucket_slots(self, edge):
        v = C.c_int()
        L.call("hfm_serve_bucket_slots", self._h, int(edge), C.byref(v))
        return v.value

    def submit(self, req):
        """Queue ``req`` (device tensors); returns its ticket."""
        sig = req.sigma.contiguous()
        rhs = req.rhs.contiguous()
        x = torch.empty((req.n,) * 3, dtype=torch.float64, device=sig.device)
        torch.cuda.current_stream().synchronize()  # the buckets read the inputs on their streams
        t = C.c_int64()
        P = lambda a: C.c_void_p(a.data_ptr())
        L.call("hfm_serve_submit", self._h, int(req.n), P(sig[0]), P(sig[1]), P(sig[2]), P(rhs),
               P(x), C.byref(t))
        self._keep[t.value] = (sig, rhs, x)
        return t.value

    def poll(self, cap=256):
        """Finished requests: a list of dicts (ticket, status, cycles, outer, rel_resid, x)."""
        buf = (L.HfmServeResult * cap)()
        n = C.c_int()
        L.call("hfm_serve_poll", self._h, buf, cap, C.byref(n))
        out = []
        for r in buf[:n.value]:
            _, _, x = self._keep.pop(r.ticket)
            out.append(dict(ticket=r.ticket, status=r.status, cycles=r.cycles, outer=r.outer,
                            rel_resid=r.rel_resid, x=x))
        return out

    def cancel(self, ticket):
        L.call("hfm_serve_cancel", self._h, int(ticket))

    def pending(self):
        q, r = C.c_int(), C.c_int()
        L.call("hfm_serve_pending", self._h, C.byref(q), C.byref(r))
        return q.value, r.value

    def serve(self, requests, timeout_s=600.0):
        """Submit every request, poll until all are reported; {ticket: result}, and the
        tickets in request order."""
        tickets = [self.submit(r) for r in requests]
        done = {}
        t0 = time.perf_counter()
        while len(done) < len(tickets):
            for r in self.poll():
                done[r["ticket"]] = r
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError("hfm_serve_poll: requests still pending after %.0f s" % timeout_s)
        return done, tickets

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().hfm_serve_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_one_at_a_time(requests, cfg=None, time_budget_s=None, keep_solutions=False):
    """The plain path: one request at a time through a single-slot float32 handle per edge.
    Returns (results, seconds)."""
    cfg = cfg or SolverConfig(cycle="V", accel="ir", storage="f32", tol=1e-6, max_cycles=600,
                              inner_tol=1e-3)
    handles = {}
    results = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in requests:
        h = handles.get(r.n)
        if h is None:
            h = handles[r.n] = Multigrid((r.n, r.n, r.n), L.OP_SIGMA7, cfg, slots=1)
        sig = r.sigma if r.sigma.is_cuda else r.sigma.cuda()
        rhs = r.rhs if r.rhs.is_cuda else r.rhs.cuda()
        ts = time.perf_counter() - t0
        h.set_operator(Sigma7(sig[0], sig[1], sig[2]))
        h.load(0, rhs)
        while True:
            h.run(cfg.cycles_per_launch)
            s = h.query()[0]
            if not s["active"]:
                break
        phi = h.fetch_f64(0) if cfg.accel == "ir" else h.fetch(0)
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        results.append(SolveResult(r.rid, r.n, s["status"], s["cycles"], s["outer"],
                                   s["rel_resid"], ts, te, te - ts,
                                   phi if keep_solutions else None))
        if time_budget_s is not None and te > time_budget_s:
            break
    dt = time.perf_counter() - t0
    for h in handles.values():
        h.close()
    return results, dt


def latency_stats(results):
    lat = np.array([r.latency for r in results]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
