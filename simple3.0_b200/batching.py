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

import ctypes as C
import dataclasses
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib
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


def _ctf_records(chunks) -> object:
    """the chunks' per-particle CTF parameters, concatenated, as the C ABI's record array"""
    n = sum(ch.nptcls for ch in chunks)
    dt = np.dtype([("smpd", np.float32), ("kv", np.float32), ("cs", np.float32), ("fraca", np.float32),
                   ("dfx", np.float32), ("dfy", np.float32), ("angast", np.float32), ("phshift", np.float32),
                   ("l_phaseplate", np.int32)])
    assert dt.itemsize == C.sizeof(_lib.CtfParams)
    rec = np.zeros(n, dt)
    o = 0
    for ch in chunks:
        s = slice(o, o + ch.nptcls)
        rec["smpd"][s], rec["kv"][s], rec["cs"][s], rec["fraca"][s] = ch.smpd, ch.kv, ch.cs, ch.fraca
        rec["dfx"][s] = ch.dfx
        rec["dfy"][s] = ch.dfx if ch.dfy is None else ch.dfy
        rec["angast"][s] = 0.0 if ch.angast is None else ch.angast
        o += ch.nptcls
    arr = (_lib.CtfParams * n)()
    C.memmove(arr, rec.ctypes.data, rec.nbytes)
    return arr


def grouped_handle(cs, device: int = 0, stream=None):
    """One handle holding the chunks cs (of one geometry): references concatenated, particles in
    consecutive slots, their CTFs; returns (handle, groups) with groups as pftcc_search_groups
    takes them, (first reference, references, first slot, particles) per chunk, 1-based."""
    import torch
    nrefs = sum(ch.nrefs for ch in cs)
    nptcls = sum(ch.nptcls for ch in cs)
    pc = polarft_corrcalc()
    try:
        c0 = cs[0]
        pc.new(nrefs, (1, nptcls), box=c0.box, nrots=c0.nrots, kfromto=(c0.kfrom, c0.kto), ctf=True,
               ctf_frame="ptcl", device=device)
        if stream is not None:
            pc.set_stream(stream)
        # the references through pinned host memory (one upload per reference set)
        refs = torch.empty((nrefs,) + tuple(np.asarray(c0.refs).shape[1:]), dtype=torch.complex64, pin_memory=True)
        r = 0
        for ch in cs:
            refs[r:r + ch.nrefs] = torch.from_numpy(np.asarray(ch.refs, np.complex64))
            r += ch.nrefs
        pc.set_refs(1, refs.numpy(), True)
        pc.set_refs(1, refs.numpy(), False)
        groups, r, s = [], 1, 1
        for ch in cs:
            if hasattr(ch.cmats, "data_ptr"):
                pc.polarize_ptcls_dev(s - 1, ch.nptcls, ch.cmats.contiguous().data_ptr())
            else:
                pc.polarize_ptcls(s - 1, np.asarray(ch.cmats))
            groups.append((r, ch.nrefs, s, ch.nptcls))
            r += ch.nrefs
            s += ch.nptcls
        pc.create_polar_absctfmats(_ctf_records(cs))
    except BaseException:
        pc.kill()
        raise
    return pc, groups


def _search_geometry(cs, precision, ntop, device, stream):
    """one geometry's chunks in one handle, searched by one pftcc_search_groups call"""
    pc, groups = grouped_handle(cs, device, stream)
    try:
        out = pc.search_groups(groups, cs[0].shifts, precision, ntop)
        res = []
        for (r0, _, s0, n) in groups:
            x = out[s0 - 1:s0 - 1 + n].copy()
            x["iref"] -= (r0 - 1) * (x["iref"] > 0)
            res.append(x)
        return res
    finally:
        pc.kill()


def search_grouped(chunks, precision: str = "bf16x3", ntop: int = 8, device: int = 0, streams: int = 3) -> list:
    """The queue as grouped searches: the chunks of each geometry (box, nrots, shells, shift list)
    go into one handle -- their references and particles concatenated -- and one
    pftcc_search_groups call searches every chunk's particles against its own references (one
    persistent tensor-core launch over all the chunks' work items per batch of waves, one
    transform launch over all their particles).  The geometries run on up to `streams` host
    threads with their own CUDA streams.  Returns each chunk's result as search_chunk does, in
    submission order."""
    import torch
    by_geom = {}
    for i, ch in enumerate(chunks):
        sh = None if ch.shifts is None else np.ascontiguousarray(ch.shifts, np.float32).reshape(-1, 2)
        key = (ch.box, ch.nrots, ch.kfrom, ch.kto, None if sh is None else sh.tobytes())
        by_geom.setdefault(key, []).append(i)
    keys = list(by_geom)
    torch.cuda.synchronize(device)      # chunk inputs made on other streams are complete
    strs = [torch.cuda.Stream(device=device) for _ in range(max(1, min(streams, len(keys))))]

    def one(k):
        st = strs[keys.index(k) % len(strs)]
        return _search_geometry([chunks[i] for i in by_geom[k]], precision, ntop, device, st.cuda_stream)

    results = [None] * len(chunks)
    with ThreadPoolExecutor(max_workers=len(strs)) as ex:
        for k, res in zip(keys, ex.map(one, keys)):
            for i, x in zip(by_geom[k], res):
                results[i] = x
    return results


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
