"""Copies between large pageable host arrays and the device.

A copy from pageable host memory goes through the driver's staging one piece at
a time on the calling thread.  For arrays of hundreds of MB and more (the
reference's per-frequency model domain is [nz][nw][ny][nx], 13 GB per
component for a 256 x 256 x 128 x 200 problem) this module stages through two
pinned buffers instead: a pool of threads copies each chunk between the
caller's array and a pinned buffer (numpy releases the GIL while it copies),
and one asynchronous copy per chunk on a side stream moves it across the host
link, so the host copies of one chunk overlap the link copy of the next.
The calling stream waits for the side stream (host to device) or the side
stream for the calling stream (device to host), so kernels and results stay
in stream order.
"""
from __future__ import annotations

import concurrent.futures
import os
import threading

import numpy as np
import torch

CHUNK_BYTES = 64 << 20        # bytes per pinned staging buffer
THRESHOLD_BYTES = 256 << 20   # arrays at least this large take the staged path

_lock = threading.Lock()
_pool = None
_state = {}  # (device index, chunk bytes) -> (side stream, [pinned buffers], [events], lock)


def _threads():
    return max(1, min(16, os.cpu_count() or 1))


def _get_pool():
    global _pool
    with _lock:
        if _pool is None:
            _pool = concurrent.futures.ThreadPoolExecutor(_threads())
        return _pool


def _get_state(device):
    idx = device.index if device.index is not None else torch.cuda.current_device()
    with _lock:
        st = _state.get((idx, CHUNK_BYTES))
        if st is None:
            with torch.cuda.device(idx):
                side = torch.cuda.Stream(idx)
                bufs = [torch.empty(CHUNK_BYTES, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
                evs = [None, None]
            st = (side, bufs, evs, threading.Lock())
            _state[(idx, CHUNK_BYTES)] = st
        return st


def host_view(a):
    """The numpy view of a host array (numpy, or a CPU tensor in pageable memory)
    that takes the staged path: C-contiguous complex64 of at least
    THRESHOLD_BYTES; else None."""
    if isinstance(a, torch.Tensor):
        if a.device.type != "cpu" or a.dtype != torch.complex64 or not a.is_contiguous() or a.is_pinned():
            return None
        a = a.numpy()
    if isinstance(a, np.ndarray) and a.dtype == np.complex64 and a.flags.c_contiguous and a.nbytes >= THRESHOLD_BYTES:
        return a
    return None


def _par_copy(dst, src):
    """dst[:] = src for two 1-D uint8 views of equal length, split over the pool."""
    n = src.size
    k = _threads()
    step = -(-n // k)
    parts = [(i, min(i + step, n)) for i in range(0, n, step)]
    if len(parts) == 1:
        np.copyto(dst, src)
        return
    list(_get_pool().map(lambda r: np.copyto(dst[r[0]:r[1]], src[r[0]:r[1]]), parts))


def to_device(a, device):
    """A complex64 device tensor holding the C-contiguous complex64 array a."""
    device = torch.device(device)
    side, bufs, evs, lock = _get_state(device)
    with lock:
        return _to_device(a, device, side, bufs, evs)


def _to_device(a, device, side, bufs, evs):
    out = torch.empty(a.shape, dtype=torch.complex64, device=device)
    src = a.reshape(-1).view(np.uint8)
    dst = out.view(-1).view(torch.uint8)
    cur = torch.cuda.current_stream(device)
    side.wait_stream(cur)  # out's memory is free to write on the side stream
    n = src.size
    for i, off in enumerate(range(0, n, CHUNK_BYTES)):
        m = min(CHUNK_BYTES, n - off)
        j = i & 1
        if evs[j] is not None:
            evs[j].synchronize()  # the link copy that last read this buffer is done
        host = bufs[j].numpy()
        _par_copy(host[:m], src[off:off + m])
        with torch.cuda.stream(side):
            dst[off:off + m].copy_(bufs[j][:m], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(side)
        evs[j] = ev
    cur.wait_stream(side)
    out.record_stream(side)
    return out


def to_host(t, a):
    """a[...] = t for a device tensor t and a writable C-contiguous complex64
    array a of the same number of elements."""
    side, bufs, evs, lock = _get_state(t.device)
    with lock:
        _to_host(t, a, side, bufs, evs)


def _to_host(t, a, side, bufs, evs):
    device = t.device
    src = t.contiguous().view(-1).view(torch.uint8)
    dst = a.reshape(-1).view(np.uint8)
    cur = torch.cuda.current_stream(device)
    side.wait_stream(cur)  # the results are written before the side stream reads them
    n = src.numel()
    offs = list(range(0, n, CHUNK_BYTES))

    def issue(i):
        off = offs[i]
        m = min(CHUNK_BYTES, n - off)
        j = i & 1
        with torch.cuda.stream(side):
            bufs[j][:m].copy_(src[off:off + m], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(side)
        evs[j] = ev

    if offs:
        issue(0)
    for i, off in enumerate(offs):
        m = min(CHUNK_BYTES, n - off)
        j = i & 1
        evs[j].synchronize()
        if i + 1 < len(offs):
            issue(i + 1)  # the other buffer: its previous chunk was copied out below
        _par_copy(dst[off:off + m], bufs[j].numpy()[:m])
    src.record_stream(side)
