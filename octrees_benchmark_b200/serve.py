"""Python front end of the serving scheduler (oct_server_* in the C ABI), the
serving workload and a client that replays a request stream in real time.

``Server`` wraps one scheduler: continuous batching over device-resident
clouds (or, with ``plain=True``, one request per launch through the single-cloud
path).  ``ServingWorkload`` holds the serving form of the benchmark: 16
device-resident clouds of 1M-50M points (generator seeds 10-25), a Poisson
stream of radius / kNN requests (seed 4) and cloud insertions.  ``replay``
submits the stream at its arrival times from one thread while a second thread
collects completions and releases them, and returns latency percentiles,
throughput and the scheduler's counters.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import capi
from .capi import (OCT_CLOUD_OWNED, OCT_SERVER_FIFO, OCT_SERVER_NO_GRAPH, OCT_SERVER_PLAIN, OctCompletion,
                   OctRequest, OctSearchConfig, OctServerParams, OctServerStats, lib)
from .engine import Request
from .linear_octree import _sync_current_stream


def _check(status: int, h, what: str) -> None:
    if status == capi.OCT_OK:
        return
    L = lib()
    msg = L.oct_status_string(status).decode()
    if h:
        buf = C.create_string_buffer(512)
        L.oct_server_last_error(h, buf, 512)
        if buf.value:
            msg += ": " + buf.value.decode()
    raise capi.OctError(status, f"{what}: {msg}")


class Server:
    """A serving scheduler on one device."""

    def __init__(self, device: int = 0, plain: bool = False, slots: int = 3, max_batch_requests: int = 1024,
                 max_batch_queries: int = 512 << 10, hbm_budget: int = 120 << 30, max_wait_ms: float = 40.0,
                 fifo: bool = False, graph: bool = True):
        L = lib()
        self._L = L
        flags = ((OCT_SERVER_PLAIN if plain else 0) | (OCT_SERVER_FIFO if fifo else 0) |
                 (0 if graph else OCT_SERVER_NO_GRAPH))
        p = OctServerParams(device, flags, slots, max_batch_requests, max_batch_queries, hbm_budget, max_wait_ms)
        h = C.c_void_p()
        _check(L.oct_server_create(C.byref(p), C.byref(h)), None, "oct_server_create")
        self._h = h
        self._keep = {}  # ticket -> request (its centre tensors stay alive until completion)
        self._lock = threading.Lock()

    def close(self):
        if getattr(self, "_h", None):
            self._L.oct_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_config(self, fp32_filter=False, knn_bucket=128, radius_blocks_per_sm=0, knn_blocks_per_sm=0,
                   serial=False, knn_group=True):
        cfg = OctSearchConfig(1, int(fp32_filter), 32, int(bool(knn_group)), int(knn_bucket))
        cfg.reserved[0], cfg.reserved[1], cfg.reserved[2] = radius_blocks_per_sm, knn_blocks_per_sm, int(serial)
        _check(self._L.oct_server_set_config(self._h, C.byref(cfg)), self._h, "oct_server_set_config")

    def add_cloud(self, oc, owned: bool = False):
        """Register a built LinearOctree; with ``owned`` the server takes the handle over (and may evict it)."""
        _check(self._L.oct_server_add_cloud(self._h, oc.handle, OCT_CLOUD_OWNED if owned else 0), self._h,
               "oct_server_add_cloud")
        if owned:
            oc._h = None  # the server destroys it

    def remove_cloud(self, handle):
        _check(self._L.oct_server_remove_cloud(self._h, handle), self._h, "oct_server_remove_cloud")

    def submit(self, req: Request, sync: bool = True) -> int:
        """Queue a request; ``sync`` waits for the current torch stream first (where its tensors were made)."""
        if sync:
            _sync_current_stream()
        r = req.to_c()
        t = C.c_uint64()
        _check(self._L.oct_server_submit(self._h, C.byref(r), C.byref(t)), self._h, "oct_server_submit")
        with self._lock:
            self._keep[t.value] = req
        return t.value

    def poll(self, max_n: int = 1024, wait_ms: int = 0):
        buf = (OctCompletion * max_n)()
        n = C.c_uint32()
        _check(self._L.oct_server_poll(self._h, buf, max_n, C.byref(n), wait_ms), self._h, "oct_server_poll")
        out = []
        for i in range(n.value):
            c = buf[i]
            out.append(dict(ticket=c.ticket, status=c.status, type=c.type, nq=c.nq, n_results=c.n_results,
                            queue_ms=c.queue_ms, latency_ms=c.latency_ms))
        return out

    def radius_result(self, ticket: int, nq: int, n_results: int):
        offs = np.zeros(nq + 1, np.uint64)
        idx = np.zeros(max(1, n_results), np.uint32)
        _check(self._L.oct_server_copy_radius(self._h, ticket, offs.ctypes.data, idx.ctypes.data, idx.shape[0], 0),
               self._h, "oct_server_copy_radius")
        return offs, idx[:n_results]

    def knn_result(self, ticket: int, nq: int, k: int):
        idx = np.zeros((nq, k), np.uint32)
        d2 = np.zeros((nq, k), np.float64)
        cnt = np.zeros(nq, np.uint32)
        _check(self._L.oct_server_copy_knn(self._h, ticket, idx.ctypes.data, d2.ctypes.data, cnt.ctypes.data, 0),
               self._h, "oct_server_copy_knn")
        return idx, d2, cnt

    def release(self, ticket: int):
        _check(self._L.oct_server_release(self._h, ticket), self._h, "oct_server_release")
        with self._lock:
            self._keep.pop(ticket, None)

    def stats(self) -> dict:
        s = OctServerStats()
        _check(self._L.oct_server_get_stats(self._h, C.byref(s)), self._h, "oct_server_get_stats")
        return {f: getattr(s, f) for f, _ in OctServerStats._fields_}


# ----------------------------------------------------------------- workload ---
SERVE_DENSITY = 10_000_000 / 1500.0 ** 2  # points per m^2 of the 10M-point 1.5 km tile


def serving_cloud_specs(n_clouds: int = 16, seed: int = 4, n_min: int = 1_000_000, n_max: int = 50_000_000):
    """Resident clouds: sizes log-uniform in [n_min, n_max] (seed), generator seeds 10, 11, ..."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_clouds):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        out.append(dict(n=n, tile_m=math.sqrt(n / SERVE_DENSITY), seed=10 + i, encoder=5, max_leaf=64,
                        n_queries=0))
    return out


@dataclass
class StreamItem:
    t: float        # arrival time (s from the start)
    cloud: int      # index into the resident clouds (or -1 - j for the j-th inserted cloud)
    kind: str       # "radius" or "knn"
    nq: int
    radius: float
    k: int


def serving_stream(rate: float = 2000.0, seconds: float = 60.0, seed: int = 4, n_clouds: int = 16,
                   max_batch: int = 100_000, insert_every: float = 10.0):
    """Poisson arrivals; each request a radius (r ~ U[0.5, 10]) or kNN (k in {10, 50, 250}) batch of
    1..max_batch centres (log-uniform) on a random resident cloud; a cloud insertion every ``insert_every``
    seconds (the inserted cloud also takes requests until the next insertion replaces it)."""
    rng = np.random.default_rng(seed)
    n = rng.poisson(rate * seconds)
    times = np.sort(rng.uniform(0.0, seconds, n))
    items = []
    for t in times:
        nq = int(min(max_batch, math.floor(math.exp(rng.uniform(0.0, math.log(max_batch + 1))))))
        nq = max(1, nq)
        epoch = int(t // insert_every) if insert_every > 0 else 0
        choices = n_clouds + (1 if epoch > 0 else 0)
        c = int(rng.integers(0, choices))
        cloud = c if c < n_clouds else -epoch  # -epoch: the cloud inserted at the start of this epoch
        if rng.random() < 0.5:
            items.append(StreamItem(float(t), cloud, "radius", nq, float(rng.uniform(0.5, 10.0)), 0))
        else:
            items.append(StreamItem(float(t), cloud, "knn", nq, 0.0, int(rng.choice([10, 50, 250]))))
    return items


class ServingWorkload:
    """Resident clouds, their centre pools, the inserted clouds' points and the request stream."""

    def __init__(self, device: int = 0, seconds: float = 60.0, rate: float = 2000.0, n_clouds: int = 16,
                 insert_every: float = 10.0, pool: int = 200_000, workers=None, cloud_points=(1_000_000, 50_000_000),
                 insert_points=(1_000_000, 10_000_000), max_batch: int = 100_000):
        import torch

        from .linear_octree import LinearOctree
        from .workloads import generate_points

        self.seconds, self.rate, self.insert_every = seconds, rate, insert_every
        self.specs = serving_cloud_specs(n_clouds, n_min=cloud_points[0], n_max=cloud_points[1])
        n_ins = int(seconds // insert_every) if insert_every > 0 else 0
        rng = np.random.default_rng(44)
        lo, hi = math.log(insert_points[0]), math.log(insert_points[1])
        self.insert_specs = [dict(n=int(round(math.exp(rng.uniform(lo, hi)))), seed=30 + j,
                                  encoder=5, max_leaf=64, n_queries=0) for j in range(n_ins)]
        for s in self.insert_specs:
            s["tile_m"] = math.sqrt(s["n"] / SERVE_DENSITY)
        t0 = time.perf_counter()
        pts = generate_points(self.specs + self.insert_specs, workers)
        self.gen_s = time.perf_counter() - t0
        self.clouds, self.pools = [], []
        g = torch.Generator(device="cuda").manual_seed(4)
        for spec, p in zip(self.specs, pts[: len(self.specs)]):
            d = torch.from_numpy(p).cuda(device)
            oc = LinearOctree(d, encoder=spec["encoder"], max_points_leaf=spec["max_leaf"], device=device)
            self.clouds.append(oc)
            self.pools.append(d[torch.randint(0, spec["n"], (pool,), device="cuda", generator=g)].contiguous())
            del d
        # the inserted clouds' points and centre pools are on the device before the stream starts, so that
        # an insertion during the stream allocates nothing outside the library's own pool
        brng = np.random.default_rng(8)
        self.insert_points, self.insert_pools = [], []
        for spec, p in zip(self.insert_specs, pts[len(self.specs):]):
            d = torch.from_numpy(p).cuda(device)
            sel = torch.from_numpy(brng.integers(0, spec["n"], pool)).cuda(device)
            self.insert_points.append(d)
            self.insert_pools.append(d[sel].contiguous())
        self.stream = serving_stream(rate, seconds, n_clouds=n_clouds, max_batch=min(max_batch, pool),
                                     insert_every=insert_every)
        self.n_points = sum(s["n"] for s in self.specs)
        self.pool = pool
        torch.cuda.synchronize()

    def describe(self) -> str:
        sizes = [s["n"] for s in self.specs]
        nq = sum(it.nq for it in self.stream)
        return (f"{len(self.specs)} resident synthetic LiDAR clouds (generator seeds 10-{9 + len(self.specs)}), "
                f"{min(sizes):,}-{max(sizes):,} points ({self.n_points:,} in all, {SERVE_DENSITY:.2f} pts/m^2), "
                f"Hilbert, leaf 64; Poisson stream of {len(self.stream):,} requests at {self.rate:g}/s for "
                f"{self.seconds:g} s (seed 4), {nq:,} centres: half radius (sphere, neighborsPrune, r ~ U[0.5, 10] m), "
                f"half kNN (k in {{10, 50, 250}}), 1-100,000 centres each (log-uniform); a 1M-10M-point cloud "
                f"inserted every {self.insert_every:g} s (the previous insert evicted); HBM budget 120 GB")


def _pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


def replay(wl: ServingWorkload, server: Server, drain_s: float = 60.0, owned_inserts: bool = True,
           insert_wait_s: float = 120.0):
    """Submit the stream at its arrival times; returns latency / throughput figures.

    Inserted clouds are built by a background thread on its own stream, each
    during the epoch before its own.  That thread waits for its own stream
    only: a device-wide synchronisation would fail while the server's
    scheduler captures a batch graph on another stream.  Every wait here is
    bounded; a failed or late insertion is reported (its requests are counted
    as skipped) instead of stalling the stream, and an error raised in a
    helper thread is re-raised here once the stream has been submitted."""
    import torch

    from .linear_octree import LinearOctree

    for oc in wl.clouds:
        server.add_cloud(oc)
    inserted = {}  # epoch -> (handle, centre pool), registered with the server
    built = {}
    failed_epochs = set()
    thread_errors = []  # (thread name, exception)
    ready = {e: threading.Event() for e in range(1, len(wl.insert_specs) + 1)}
    dev = torch.cuda.current_device()

    def builder():
        bstream = torch.cuda.Stream(device=dev)
        try:
            for e in range(1, len(wl.insert_specs) + 1):
                d, pool, spec = wl.insert_points[e - 1], wl.insert_pools[e - 1], wl.insert_specs[e - 1]
                try:
                    with torch.cuda.stream(bstream):
                        oc = LinearOctree(d, encoder=spec["encoder"], max_points_leaf=spec["max_leaf"], device=dev)
                    bstream.synchronize()  # this stream only: never the device
                    built[e] = (oc, pool)
                except Exception as exc:  # noqa: BLE001 - reported with the figures
                    thread_errors.append(("insert builder", exc))
                    failed_epochs.add(e)
                finally:
                    ready[e].set()
        finally:
            for ev in ready.values():
                ev.set()

    removers = []
    bt = threading.Thread(target=builder, daemon=True)
    bt.start()
    lat, qms, nq_done = [], [], [0]
    info = {}  # ticket -> request class, for the latency split by class
    done_lat = []  # (ticket, latency) of every completion
    errors = [0]
    done_evt = threading.Event()
    skipped = [0]
    n_total = len(wl.stream)

    def collector():
        got = 0
        try:
            while got + skipped[0] < n_total and not done_evt.is_set():
                for c in server.poll(4096, wait_ms=5):
                    got += 1
                    if c["status"] != capi.OCT_OK:
                        errors[0] += 1
                    else:
                        lat.append(c["latency_ms"])
                        qms.append(c["queue_ms"])
                        nq_done[0] += c["nq"]
                        done_lat.append((c["ticket"], c["latency_ms"]))
                    server.release(c["ticket"])
        except Exception as exc:  # noqa: BLE001
            thread_errors.append(("collector", exc))
        finally:
            done_evt.set()

    def remover(old):
        try:
            server.remove_cloud(C.c_void_p(old))
        except Exception as exc:  # noqa: BLE001
            thread_errors.append(("remover", exc))

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    rng = np.random.default_rng(7)
    t0 = time.perf_counter()
    late = []
    try:
        for it in wl.stream:
            if done_evt.is_set() and thread_errors:
                break  # the collector died: nothing would be collected
            epoch = int(it.t // wl.insert_every) if wl.insert_every > 0 else 0
            if epoch > 0 and epoch not in inserted and epoch not in failed_epochs:
                # insert this epoch's cloud, evict the previous one
                if not ready[epoch].wait(timeout=insert_wait_s) or epoch not in built:
                    failed_epochs.add(epoch)
                else:
                    oc, pool = built.pop(epoch)
                    h = oc.handle.value
                    server.add_cloud(oc, owned=owned_inserts)
                    inserted[epoch] = (h, pool)
                    if epoch - 1 in inserted:  # removed once its requests have finished, off the submit thread
                        old = inserted.pop(epoch - 1)[0]
                        rt = threading.Thread(target=remover, args=(old,), daemon=True)
                        rt.start()
                        removers.append(rt)
            now = time.perf_counter() - t0
            if it.t > now:
                time.sleep(it.t - now)
            late.append(max(0.0, time.perf_counter() - t0 - it.t))
            if it.cloud >= 0:
                handle, pool = wl.clouds[it.cloud].handle, wl.pools[it.cloud]
            elif -it.cloud in inserted:
                handle, pool = inserted[-it.cloud]
            else:  # its cloud's insertion failed
                skipped[0] += 1
                continue
            off = int(rng.integers(0, wl.pool - it.nq + 1))
            centres = pool[off: off + it.nq]
            proxy = _Handle(handle)
            if it.kind == "radius":
                req = Request(proxy, "radius", centres, radius=it.radius, kernel="sphere", algo="neighborsPrune")
            else:
                req = Request(proxy, "knn", centres, k=it.k)
            size = "centres<=1k" if it.nq <= 1000 else ("centres<=10k" if it.nq <= 10_000 else "centres>10k")
            kind = f"knn k={it.k}" if it.kind == "knn" else ("radius r<=5" if it.radius <= 5.0 else "radius r>5")
            cl = f"{kind}, {size}"
            t = server.submit(req, sync=False)  # the pools were complete before the stream started
            info[t] = cl
    finally:
        t_sub = time.perf_counter() - t0
        th.join(timeout=max(1.0, drain_s))
        done_evt.set()
        th.join(timeout=5.0)
        t_end = time.perf_counter() - t0
        for rt in removers:
            rt.join(timeout=5.0)
        bt.join(timeout=5.0)
    if thread_errors:
        name, exc = thread_errors[0]
        raise RuntimeError(f"serving replay: the {name} thread failed: {exc!r}") from exc
    st = server.stats()
    completed = len(lat)
    cls_lat = {}
    for t, v in done_lat:
        cl = info.get(t)
        if cl is not None:
            cls_lat.setdefault(cl, []).append(v)
    return {
        "requests": n_total, "completed": completed, "errors": errors[0],
        "unfinished": n_total - completed - errors[0] - skipped[0], "skipped": skipped[0],
        "p50_ms": _pct(lat, 50), "p90_ms": _pct(lat, 90), "p99_ms": _pct(lat, 99), "max_ms": max(lat) if lat else None,
        "queue_p50_ms": _pct(qms, 50), "queue_p99_ms": _pct(qms, 99),
        "queries_completed": nq_done[0], "wall_s": t_end, "submit_s": t_sub,
        "qps": nq_done[0] / t_end if t_end > 0 else None,
        "submit_lag_p99_ms": 1e3 * _pct(late, 99) if late else None,
        "batches": st["batches"], "admission_stalls": st["admission_stalls"],
        "max_submit_ms": st["max_submit_ms"], "max_finish_ms": st["max_finish_ms"],
        "budget_evictions": st["evictions"], "clouds_inserted": len(inserted) + len(removers),
        "insert_failures": len(failed_epochs), "clouds_removed": len(removers), "peak_budget_bytes": st["peak_bytes"],
        "by_class": {k: {"requests": len(v), "p50_ms": _pct(v, 50), "p99_ms": _pct(v, 99)}
                     for k, v in sorted(cls_lat.items())},
    }


class _Handle:
    """A stand-in exposing ``.handle`` for a raw cloud handle."""

    def __init__(self, h):
        self.handle = h if isinstance(h, C.c_void_p) else C.c_void_p(h)
