"""Background wavefields of a run kept in files, depth by depth, in the layout of
the reference's checkpoint store.

The reference's ``WavefieldPool`` (``propagator/src/WavefieldPool.cpp:13-219``)
ZFP-compresses every depth slice of a background wavefield at the fixed rate
``compress_rate`` on host threads and writes it with ``pwrite`` into one file
per tag, ``<wfld_path>/<run_id>/checkpoints_<tag>.bin``, each depth a chunk of
fixed size (``zfp_stream_maximum_size``) at offset ``iz * chunk``
(``:60-61, :78-100``); depth slices are read back with ``pread`` and
decompressed (``decompress_slice_async``).  This store keeps the same file
layout and keys (``wfld_path``, ``compress_rate``, ``wflds_to_store``) with
this library's codecs in place of ZFP, which is not available to reproduce:

* ``compress_rate = 8`` or ``16``: the fixed-rate packed format of
  ``fwix_pack_wavefield`` (8.5 or 16.5 bits per value; chunk =
  ``fwix_plan_packed_bytes``), packed on the device straight into a pinned host
  buffer;
* no ``compress_rate``: complex64 as is (chunk = the wavefield's bytes).

Writes run on a host thread pool after the device-to-host copy of their slice
has finished (a CUDA event per buffer), with ``wflds_to_store`` pinned buffers in
flight, as the reference pipelines its compression; reads fill a pinned buffer
with ``pread`` and unpack (or copy) it into a device wavefield on the current
stream.  The files are plain byte arrays: a later process with the same plan
geometry can read them back (``load``), which is what a restart needs.
"""
from __future__ import annotations

import os
import tempfile
from concurrent.futures import ThreadPoolExecutor

import torch

from . import _lib as L
from .plan import _p, _stream


def _get(par, key, default=None):
    if par is None:
        return default
    v = par.get(key, default) if hasattr(par, "get") else getattr(par, key, default)
    return default if v is None else v


class WavefieldPool:
    """Depth slices [ns][nw][NY][NX] of one plan's wavefields, per tag, in files."""

    def __init__(self, plan, par, run_id, max_depth):
        self.plan = plan
        rate = _get(par, "compress_rate")
        if rate is not None and float(rate) not in (8.0, 16.0):
            raise ValueError(f"compress_rate {rate} is not supported: the packed store has rates 8 and 16")
        self.packed = rate is not None
        if self.packed and int(float(rate)) != getattr(plan, "pack_bits", 8):
            plan.set_pack_rate(int(float(rate)))
        self.wbytes = int(torch.Size(plan.wshape).numel()) * 8
        self.chunk = plan.packed_bytes if self.packed else self.wbytes
        self.max_depth = int(max_depth)
        self.base = os.path.join(str(_get(par, "wfld_path", tempfile.gettempdir())), str(run_id))
        os.makedirs(self.base, exist_ok=True)
        n = max(1, int(_get(par, "wflds_to_store", 3)))
        self.buffers = [torch.empty(self.chunk, dtype=torch.uint8, pin_memory=True) for _ in range(n)]
        self.events = [None] * n
        self.pending = [None] * n
        self.next = 0
        self.io = ThreadPoolExecutor(max_workers=n)
        self.fds = {}
        self.written = 0

    def path(self, tag):
        return os.path.join(self.base, f"checkpoints_{tag}.bin")

    def _fd(self, tag):
        if tag not in self.fds:
            fd = os.open(self.path(tag), os.O_CREAT | os.O_RDWR | os.O_TRUNC, 0o664)
            try:
                os.posix_fallocate(fd, 0, self.max_depth * self.chunk)
            except (AttributeError, OSError):
                os.ftruncate(fd, self.max_depth * self.chunk)
            self.fds[tag] = fd
        return self.fds[tag]

    def _free_buffer(self):
        i = self.next
        self.next = (i + 1) % len(self.buffers)
        if self.pending[i] is not None:
            self.pending[i].result()        # its previous write has finished
            self.pending[i] = None
        return i

    def compress_slice(self, iz, wfld, tag):
        """Stores depth iz of ``wfld`` (a device wavefield) under ``tag``: packed (or
        copied) into a pinned buffer on the current stream, written to the tag's
        file at offset iz * chunk by a host thread once the copy has finished."""
        if not 0 <= iz < self.max_depth:
            raise IndexError(f"depth {iz} outside [0, {self.max_depth})")
        fd = self._fd(tag)
        i = self._free_buffer()
        buf = self.buffers[i]
        if self.packed:
            L.check(self.plan.lib.fwix_pack_wavefield(self.plan._h, _p(wfld), _p(buf), _stream()))
        else:
            buf.copy_(wfld.reshape(-1).view(torch.uint8), non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        mv = buf.numpy()

        def write():
            ev.synchronize()
            view = memoryview(mv)
            off = 0
            while off < len(view):
                off += os.pwrite(fd, view[off:], iz * self.chunk + off)
            return off
        self.pending[i] = self.io.submit(write)
        self.written += self.chunk

    def decompress_slice(self, iz, tag, out):
        """Reads depth iz of ``tag`` into the device wavefield ``out`` (waits for
        the pool's pending writes first)."""
        self.wait_to_finish()
        if tag not in self.fds and not os.path.exists(self.path(tag)):
            raise FileNotFoundError(self.path(tag))
        fd = self.fds.get(tag)
        own = fd is None
        if own:
            fd = os.open(self.path(tag), os.O_RDONLY)
        try:
            i = self._free_buffer()
            buf = self.buffers[i]
            view = memoryview(buf.numpy())
            got = 0
            while got < self.chunk:
                n = os.preadv(fd, [view[got:]], iz * self.chunk + got)
                if n <= 0:
                    raise IOError(f"{self.path(tag)}: depth {iz} is not stored")
                got += n
        finally:
            if own:
                os.close(fd)
        if self.packed:
            L.check(self.plan.lib.fwix_unpack_wavefield(self.plan._h, _p(buf), _p(out), _stream()))
        else:
            out.reshape(-1).view(torch.uint8).copy_(buf, non_blocking=True)
        # the buffer is reused only after this stream's work on it has finished
        ev = torch.cuda.Event()
        ev.record()
        self.pending[i] = self.io.submit(ev.synchronize)
        return out

    def store(self, fields, tag):
        """Every depth of ``fields`` under ``tag``: wavefields [nz][ns][nw][NY][NX]
        (packed or copied by compress_slice), or, for a packed pool, storage that
        is already packed, [nz][packed_bytes] uint8 (device or pinned host), written
        as it is."""
        if fields.dtype == torch.uint8:
            if not self.packed or fields.shape[-1] != self.chunk:
                raise ValueError("packed storage needs a pool with compress_rate 8 and the plan's packed size")
            fd = self._fd(tag)
            for iz in range(fields.shape[0]):
                i = self._free_buffer()
                buf = self.buffers[i]
                buf.copy_(fields[iz], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record()
                mv = buf.numpy()

                def write(ev=ev, mv=mv, iz=iz):
                    ev.synchronize()
                    view = memoryview(mv)
                    off = 0
                    while off < len(view):
                        off += os.pwrite(fd, view[off:], iz * self.chunk + off)
                    return off
                self.pending[i] = self.io.submit(write)
                self.written += self.chunk
            return
        for iz in range(fields.shape[0]):
            self.compress_slice(iz, fields[iz], tag)

    def load(self, tag, out=None, host=False):
        """Every depth of ``tag`` as packed storage [nz][packed_bytes] (device, or
        pinned host memory with ``host``) for ``Plan.born_packed``; raw stores
        return complex64 wavefields [nz][ns][nw][NY][NX] on the device."""
        self.wait_to_finish()
        nz = self.max_depth
        if self.packed:
            dst = out if out is not None else self.plan.packed(nz, host=host)
            with open(self.path(tag), "rb") as f:
                for iz in range(nz):
                    f.seek(iz * self.chunk)
                    row = torch.frombuffer(bytearray(f.read(self.chunk)), dtype=torch.uint8)
                    dst[iz].copy_(row)
            return dst
        dst = out if out is not None else torch.empty((nz,) + self.plan.wshape, dtype=torch.complex64,
                                                      device=self.plan.device)
        for iz in range(nz):
            self.decompress_slice(iz, tag, dst[iz])
        return dst

    def get_total_compressed_size(self):
        """Bytes written to the files so far."""
        return self.written

    def wait_to_finish(self):
        for i, f in enumerate(self.pending):
            if f is not None:
                f.result()
                self.pending[i] = None

    def close(self):
        self.wait_to_finish()
        for fd in self.fds.values():
            os.close(fd)
        self.fds = {}
        self.io.shutdown(wait=True)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
