"""Map-making request server: independent GLS solves on one GPU, with
continuous batching.

Requests name a dataset (a pointing, a noise model and a sky signal) and a
noise realisation.  Datasets stay resident on the device once built: their
pointing (compressed indices, FP32 weights, P^T bins), their Toeplitz tile
plans and spectra (FP64 and FP32) and their block-Jacobi preconditioner
(kept with the pointing by the library after the first solve).  A request
runs in one of `slots` worker slots, each with its own CUDA stream and
library context, so the kernels of up to `slots` solves overlap on the GPU;
a request that arrives while others run is admitted as soon as a slot is
free and its working memory fits the HBM budget (first fit in arrival order,
so a small request does not wait behind a large one that does not fit yet,
and a request that waited longer than `max_bypass_s` stops later ones from
passing it).  Datasets beyond the dataset budget are evicted least recently
used when not in use.

The scheduler (Server) does not touch the GPU itself: it drives an executor
with prepare(spec) -> dataset, run(dataset, request) -> Result and
work_bytes(spec).  GpuExecutor is the one that solves; tests drive the
scheduler with a fake executor on the CPU.

There is no counterpart in the reference (MAPPRAISER's MLmap is one solve per
call, mappraiser/src/mappraiser.c:34-385); each request is that solve.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np


# --------------------------------------------------------------------------- requests
@dataclass(frozen=True)
class DatasetSpec:
    """A map-making dataset: detectors, samples, flat-sky grid, noise model."""
    key: str
    n_det: int
    n_samp: int
    width: int
    height: int
    lam: int
    fknee: float
    gap_frac: float = 0.01
    seed: int = 0

    @property
    def n_samples(self) -> int:
        return self.n_det * self.n_samp


@dataclass
class Request:
    rid: int
    spec: DatasetSpec
    noise_seed: int
    precision: str = "mixed"       # "mixed" or "fp64"
    tol: float = 1e-8
    maxiter: int = 500
    t_arrival: float = 0.0          # set by Server.submit


@dataclass
class Result:
    rid: int
    key: str
    precision: str
    x: np.ndarray | None
    lstid: np.ndarray | None
    iterations: int
    converged: bool
    n_samples: int
    t_arrival: float = 0.0
    t_start: float = 0.0
    t_end: float = 0.0
    error: str | None = None

    @property
    def latency(self) -> float:
        return self.t_end - self.t_arrival


class Ticket:
    """Handle of a submitted request."""

    def __init__(self, req: Request):
        self.request = req
        self._done = threading.Event()
        self.result: Result | None = None

    def set(self, res: Result):
        self.result = res
        self._done.set()

    def wait(self, timeout: float | None = None) -> Result:
        if not self._done.wait(timeout):
            raise TimeoutError(f"request {self.request.rid} not done")
        return self.result


# --------------------------------------------------------------------------- scheduler
@dataclass
class _Resident:
    spec: DatasetSpec
    data: object
    nbytes: int
    users: int = 0
    last_used: float = 0.0
    lock: threading.Lock = field(default_factory=threading.Lock)


class Server:
    def __init__(self, executor, slots: int = 4, work_budget: int = 64 << 30, dataset_budget: int = 64 << 30,
                 max_bypass_s: float = 2.0):
        if slots < 1:
            raise ValueError("slots >= 1")
        self.ex = executor
        self.slots = slots
        self.work_budget = work_budget
        self.dataset_budget = dataset_budget
        self.max_bypass_s = max_bypass_s
        self._cv = threading.Condition()
        self._queue: list[Ticket] = []
        self._work_used = 0
        self._running = 0
        self._resident: dict[str, _Resident] = {}
        self._closing = False
        self.max_running = 0
        self.peak_work = 0
        self.completed: list[Result] = []
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True) for i in range(slots)]
        for t in self._threads:
            t.start()

    # ---- public
    def submit(self, req: Request, t_arrival: float | None = None) -> Ticket:
        req.t_arrival = time.perf_counter() if t_arrival is None else t_arrival
        if self.ex.work_bytes(req.spec) > self.work_budget:
            raise ValueError(f"request {req.rid} needs more working memory than the whole budget")
        tk = Ticket(req)
        with self._cv:
            if self._closing:
                raise RuntimeError("server is closed")
            self._queue.append(tk)
            self._cv.notify_all()
        return tk

    def preload(self, spec: DatasetSpec):
        """Builds a dataset's resident state before requests arrive."""
        with self._cv:
            r = self._resident.get(spec.key)
            if r is not None:
                return
        data = self.ex.prepare(spec)
        with self._cv:
            self._resident.setdefault(spec.key, _Resident(spec, data, self.ex.data_bytes(data), 0,
                                                          time.perf_counter()))
            self._evict_locked()

    def close(self):
        with self._cv:
            self._closing = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for r in self._resident.values():
            self.ex.release(r.data)
        self._resident.clear()

    def resident_keys(self):
        with self._cv:
            return sorted(self._resident)

    # ---- internals
    def _pick_locked(self) -> Ticket | None:
        """First request in arrival order whose working memory fits; a request
        that has waited longer than max_bypass_s blocks the ones behind it."""
        now = time.perf_counter()
        for tk in self._queue:
            need = self.ex.work_bytes(tk.request.spec)
            if self._work_used + need <= self.work_budget:
                return tk
            if now - tk.request.t_arrival > self.max_bypass_s:
                return None
        return None

    def _evict_locked(self):
        total = sum(r.nbytes for r in self._resident.values())
        if total <= self.dataset_budget:
            return
        for r in sorted(self._resident.values(), key=lambda r: r.last_used):
            if total <= self.dataset_budget:
                break
            if r.users == 0:
                del self._resident[r.spec.key]
                self.ex.release(r.data)
                total -= r.nbytes

    def _acquire_dataset(self, spec: DatasetSpec) -> _Resident:
        with self._cv:
            r = self._resident.get(spec.key)
            if r is not None:
                r.users += 1
                return r
        data = self.ex.prepare(spec)
        with self._cv:
            r = self._resident.get(spec.key)
            if r is None:
                r = _Resident(spec, data, self.ex.data_bytes(data))
                self._resident[spec.key] = r
            else:
                self.ex.release(data)
            r.users += 1
            return r

    def _release_dataset(self, r: _Resident):
        with self._cv:
            r.users -= 1
            r.last_used = time.perf_counter()
            self._evict_locked()

    def _worker(self, slot: int):
        self.ex.start_slot(slot)
        try:
            while True:
                with self._cv:
                    tk = None
                    while True:
                        tk = self._pick_locked()
                        if tk is not None or (self._closing and not self._queue):
                            break
                        self._cv.wait(0.05)
                    if tk is None:
                        return
                    self._queue.remove(tk)
                    need = self.ex.work_bytes(tk.request.spec)
                    self._work_used += need
                    self._running += 1
                    self.max_running = max(self.max_running, self._running)
                    self.peak_work = max(self.peak_work, self._work_used)
                req = tk.request
                t_start = time.perf_counter()
                try:
                    r = self._acquire_dataset(req.spec)
                    try:
                        with r.lock:  # requests on one dataset share its device state
                            res = self.ex.run(slot, r.data, req)
                    finally:
                        self._release_dataset(r)
                except Exception as e:  # noqa: BLE001 - reported in the result
                    res = Result(req.rid, req.spec.key, req.precision, None, None, 0, False, req.spec.n_samples,
                                 error=f"{type(e).__name__}: {e}")
                res.t_arrival, res.t_start, res.t_end = req.t_arrival, t_start, time.perf_counter()
                with self._cv:
                    self._work_used -= need
                    self._running -= 1
                    self.completed.append(res)
                    self._cv.notify_all()
                tk.set(res)
        finally:
            self.ex.stop_slot(slot)


def latency_stats(results: list[Result]) -> dict:
    ok = [r for r in results if r.error is None]
    if not ok:
        return {"n": 0}
    lat = np.array([r.latency for r in ok])
    t0 = min(r.t_arrival for r in ok)
    t1 = max(r.t_end for r in ok)
    return {"n": len(ok), "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "solves_per_s": len(ok) / (t1 - t0) if t1 > t0 else float("nan"),
            "makespan_s": t1 - t0, "converged": sum(1 for r in ok if r.converged),
            "iterations_mean": float(np.mean([r.iterations for r in ok]))}


# --------------------------------------------------------------------------- workload
def _well_posed_grid(side: int, n_samples: int, min_hits: int = 16):
    """The synthetic scan needs enough samples per pixel and polarisation
    angles that change between visits: the grid side is clipped so that pixels
    get min_hits samples on average, and the height is nudged (a few rows) so
    that the scan's revisit period of width*height samples is not close to a
    multiple of the 25-sample half-wave-plate period (100 Hz sampling, 2 Hz
    rotation), where a lone detector would see one angle per pixel and the
    rcond cut would remove every pixel."""
    side = max(64, min(side, int(math.sqrt(n_samples / (min_hits * 0.75)))))
    width, height = side, max(1, (3 * side) // 4)
    period = int(round(synth_fs() / (2.0 * synth_fhwp())))
    if width % period == 0:
        width += 1
    for _ in range(period):
        k = (width * height) % period
        if min(k, period - k) >= 3:
            break
        height += 1
    return width, height


def synth_fs() -> float:
    from midapack_b200 import synth
    return synth.FS


def synth_fhwp() -> float:
    from midapack_b200 import synth
    return synth.F_HWP


def draw_specs(n: int, seed: int, max_samples: int = 1 << 28) -> list[DatasetSpec]:
    """Datasets drawn as the serving configuration: log-uniform detectors 1-32,
    samples per detector 2^18-2^23, grid side 64-1024 (4:3), lambda 2^8-2^14;
    f_knee uniform in 0.1-5 Hz; 1 % flagged samples.  The grid is then made
    well posed for the synthetic scan (_well_posed_grid)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        n_det = int(round(math.exp(rng.uniform(0.0, math.log(32.0)))))
        n_samp = int(round(2.0 ** rng.uniform(18.0, 23.0)))
        side = int(round(math.exp(rng.uniform(math.log(64.0), math.log(1024.0)))))
        lam = int(round(2.0 ** rng.uniform(8.0, 14.0)))
        fknee = float(rng.uniform(0.1, 5.0))
        n_det = max(1, min(n_det, max_samples // n_samp))
        width, height = _well_posed_grid(side, n_det * n_samp)
        out.append(DatasetSpec(f"ds{i}", n_det, n_samp, width, height, lam, fknee, 0.01, seed * 1000 + i))
    return out


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival offsets (seconds) of n requests of a Poisson stream."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def run_stream(server: Server, requests: list[Request], offsets: np.ndarray, timeout: float = 600.0) -> list[Result]:
    """Submits requests at their arrival offsets (latency counts from the
    scheduled arrival, so a late submission shows as latency) and waits for all."""
    t0 = time.perf_counter()
    tickets = []
    for req, off in zip(requests, offsets):
        now = time.perf_counter() - t0
        if off > now:
            time.sleep(off - now)
        tickets.append(server.submit(req, t_arrival=t0 + off))
    return [tk.wait(timeout) for tk in tickets]


# --------------------------------------------------------------------------- GPU executor
class GpuExecutor:
    """Builds datasets on the device and solves requests with the library
    (gls_solve_mixed or gls_solve), one CUDA stream and context per slot."""

    def __init__(self, device: int = 0, keep_maps=True):
        """keep_maps: True, False, or a predicate on the request id (maps copied to the host)."""
        import torch
        import midapack_b200 as mb
        self.torch = torch
        self.mb = mb
        self.device = device
        self.keep_maps = keep_maps
        self._slot = {}
        self._prep_lock = threading.Lock()

    # dataset bytes: pix 12, weights 24, signal 8, compressed offsets 4,
    # FP32 weights 12 and P^T bins 4 bytes per sample, plus spectra
    @staticmethod
    def work_bytes(spec: DatasetSpec) -> int:
        # per solve: two FP64 and two FP32 TOD buffers, the FP64 noise copy,
        # the FP32 noise realisation, map-domain vectors
        m = spec.n_samples
        return m * (8 * 2 + 4 * 2 + 8 + 4) + spec.width * spec.height * 3 * 8 * 12

    @staticmethod
    def data_bytes(data) -> int:
        return data["bytes"]

    def start_slot(self, slot: int):
        torch = self.torch
        torch.cuda.set_device(self.device)
        st = torch.cuda.Stream()
        with torch.cuda.stream(st):
            ctx = self.mb.Context(self.device)
        self._slot[slot] = (st, ctx)

    def stop_slot(self, slot: int):
        st, ctx = self._slot.pop(slot)
        ctx.close()

    def prepare(self, spec: DatasetSpec):
        torch, mb = self.torch, self.mb
        from midapack_b200 import synth
        with self._prep_lock:
            torch.cuda.set_device(self.device)
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                wl = synth.make_workload_torch(spec.key, spec.width, spec.height, spec.n_det, spec.n_samp,
                                               spec.n_samp, spec.lam, spec.fknee, spec.seed, spec.gap_frac)
                ctx = mb.Context(self.device)
                P = mb.Pointing(ctx, wl.pix, wl.weights, wl.n_samples, 3)
                N = mb.Noise(ctx, wl.block_sizes, wl.lam, wl.invtt)
                # one short solve builds what later solves reuse: the block-Jacobi
                # preconditioner and cut, the FP32 weights and tile plan, the P^T bins
                mb.gls_solve_mixed(ctx, P, N, wl.signal, torch.zeros_like(wl.signal), tol=1e-8, maxiter=1)
                st.synchronize()
            m = spec.n_samples
            nbytes = m * (12 + 24 + 8 + 4 + 12 + 4) + N.tile()["n_tiles"] * 16 * 1024
            return {"wl": wl, "P": P, "N": N, "ctx": ctx, "bytes": nbytes, "warm": False}

    def release(self, data):
        data["P"].close()
        data["N"].close()
        data["ctx"].close()
        data.clear()

    def run(self, slot: int, data, req: Request) -> Result:
        torch, mb = self.torch, self.mb
        from midapack_b200 import synth
        st, ctx = self._slot[slot]
        spec = req.spec
        with torch.cuda.stream(st):
            wl = data["wl"]
            noise = synth.mc_noise_torch(spec.n_det, spec.n_samp, 1, spec.fknee, seed=req.noise_seed)[0].double()
            if req.precision == "mixed":
                x, lst, cond, hits, res, info = mb.gls_solve_mixed(ctx, data["P"], data["N"], wl.signal, noise,
                                                                   tol=req.tol, maxiter=req.maxiter)
            elif req.precision == "fp64":
                x, lst, cond, hits, res, info = mb.gls_solve(ctx, data["P"], data["N"], wl.signal, noise,
                                                             tol=req.tol, maxiter=req.maxiter)
            else:
                raise ValueError(req.precision)
            keep = self.keep_maps(req.rid) if callable(self.keep_maps) else self.keep_maps
            xm = x.cpu().numpy() if keep else None
            lm = lst.cpu().numpy() if keep else None
            st.synchronize()
        return Result(req.rid, spec.key, req.precision, xm, lm, info.iterations, bool(info.converged), spec.n_samples)
