"""A streaming queue of search chunks: the batching workload of a 2D classification run,
where particle chunks of different geometries (box, nrots, shells) and sizes arrive one
after another and each is searched against its own references.

Each chunk runs through its own ``polarft_corrcalc`` handle (gridding of the particles'
half-plane FTs, |CTF| matrices, the m-domain search with the top-8 re-score), so its
result is exactly the result of searching that chunk alone.  Chunks are spread over
``workers`` host threads, each with its own CUDA stream, so that the small chunks of a
queue overlap on the GPU instead of running one after another (the library's calls
release the interpreter lock while they run).
"""
from __future__ import annotations

import dataclasses
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .pftcc import ctfparams_array, polarft_corrcalc


@dataclasses.dataclass
class Chunk:
    """One chunk of the queue.  refs: complex64 (nrefs, K, P) reference polar FTs;
    cmats: the particles' half-plane FTs, complex64 (n, box, box//2+1), a torch tensor on
    the queue's device or a host array; dfx/dfy/angast: per-particle CTF parameters."""
    box: int
    nrots: int
    kfrom: int
    kto: int
    refs: np.ndarray
    cmats: object
    dfx: np.ndarray
    dfy: np.ndarray
    angast: np.ndarray
    smpd: float = 1.3
    kv: float = 300.0
    cs: float = 2.7
    fraca: float = 0.1
    shifts: np.ndarray | None = None

    @property
    def nptcls(self) -> int:
        return int(self.cmats.shape[0])

    @property
    def nrefs(self) -> int:
        return int(self.refs.shape[0])

    def evals(self) -> float:
        ns = 1 if self.shifts is None else len(self.shifts)
        return float(self.nrefs) * self.nptcls * ns * self.nrots


def search_chunk(ch: Chunk, precision: str = "bf16x3", ntop: int = 8, device: int = 0, stream=None) -> np.ndarray:
    """Search one chunk (particle frame) and return its best (iref, irot, ishift, corr) per particle."""
    pc = polarft_corrcalc()
    try:
        pc.new(ch.nrefs, (1, ch.nptcls), box=ch.box, nrots=ch.nrots, kfromto=(ch.kfrom, ch.kto), ctf=True,
               ctf_frame="ptcl", device=device)
        if stream is not None:
            pc.set_stream(stream)
        pc.set_refs(1, ch.refs, True)
        pc.set_refs(1, ch.refs, False)
        if hasattr(ch.cmats, "data_ptr"):
            pc.polarize_ptcls_dev(0, ch.nptcls, ch.cmats.contiguous().data_ptr())
        else:
            pc.polarize_ptcls(0, np.asarray(ch.cmats))
        pc.create_polar_absctfmats(ctfparams_array(ch.nptcls, smpd=ch.smpd, kv=ch.kv, cs=ch.cs, fraca=ch.fraca,
                                                   dfx=ch.dfx, dfy=ch.dfy, angast=ch.angast))
        return pc.search_best(ch.shifts, precision, ntop=ntop)
    finally:
        pc.kill()


class SearchQueue:
    """Runs a list of chunks over ``workers`` host threads, each with its own CUDA stream;
    results come back in submission order."""

    def __init__(self, device: int = 0, precision: str = "bf16x3", ntop: int = 8, workers: int = 2):
        self.device, self.precision, self.ntop, self.workers = device, precision, ntop, max(1, workers)
        self._streams = None
        self._local = threading.local()

    def _stream(self):
        import torch
        if self._streams is None:
            self._streams = [torch.cuda.Stream(device=self.device) for _ in range(self.workers)]
            self._next = 0
            self._lock = threading.Lock()
        if not hasattr(self._local, "stream"):
            with self._lock:
                self._local.stream = self._streams[self._next % self.workers]
                self._next += 1
        return self._local.stream

    def _one(self, ch: Chunk):
        s = self._stream()
        return search_chunk(ch, self.precision, self.ntop, self.device, s.cuda_stream)

    def run(self, chunks) -> list:
        import torch
        torch.cuda.synchronize(self.device)      # chunk inputs made on other streams are complete
        with ThreadPoolExecutor(max_workers=self.workers) as ex:
            return list(ex.map(self._one, chunks))


GEOMETRIES = {"A": "config0", "B": "config1", "C": "geometry_c"}   # box 64 / 128 / 200


def synthetic_chunk(geometry: str, nrefs: int, nptcls: int, seed: int, device: str = "cuda",
                    ref_cache: dict | None = None) -> Chunk:
    """A chunk of the given geometry ("A": box 64 / nrots 128 / k 2..20, "B": box 128 /
    nrots 360 / k 2..40, "C": box 200 / nrots 600 / k 2..60) with seeded particles made as
    in the synthetic workloads (no shift search).  With ref_cache (a dict kept by the
    caller) the chunks of one geometry share one seeded set of 300 references, of which a
    chunk takes the first nrefs, as the chunks of one classification run share theirs."""
    from . import synth
    make = getattr(synth, GEOMETRIES[geometry])
    if ref_cache is not None:
        if geometry not in ref_cache:
            w0 = make(nrefs=max(300, nrefs), nptcls=1, shift_grid=())
            ref_cache[geometry] = synth.make_refs(w0)
        refs_all, R_all = ref_cache[geometry]
        refs, R = refs_all[:nrefs], R_all[:nrefs]
    w = make(nrefs=nrefs, nptcls=nptcls, seed_base=10_000 * (seed + 1), shift_grid=())
    if ref_cache is None:
        refs, R = synth.make_refs(w)
    parts = synth.make_particles(w, R, device=device)
    return Chunk(w.box, w.nrots, w.kfrom, w.kto, refs.numpy(), parts.cmat.contiguous(), parts.dfx, parts.dfy,
                 parts.angast, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca)
