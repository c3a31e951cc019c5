"""Key-sharded window-1 evolution (no counterpart in the reference, whose evolve!
runs in one process; spv_kernels.jl:3-5 names a multi-device engine as future
work).

The live set is split over R = 2^rank_bits ranks by owner(P), rank_bits
GF(2)-linear parities of the key (the bucket hash of the bucketed rotations with
other rows).  Linearity makes owner(P xor M) = owner(P) xor owner(M): the sin
branches of rank r's terms all belong to rank r xor owner(M), so a rotation is a
pairwise exchange between fixed rank pairs, not an all-to-all.  Per rotation
every rank

  1. packs the local terms that anticommute with G and survive the early-merge
     pre-filter (pp_shard_send) and swaps them with its partner rank;
  2. takes the partner's terms as foreign terms of its buckets (pp_shard_recv);
  3. rotates (pp_shard_rotate): own outputs of its terms, each summed with the
     partner's sin branch when the partner term exists, and the sin branches of
     foreign terms whose partner is absent here;

and all ranks agree on the global counts: the early-merge rule of
spv_evolve.jl:356-362 (pref = global n > append capacity) and when to give
every rank's buckets one more bit.  The union of the shards is the reference's
vector bit for bit: every output key still sums the same one or two terms.

`run_sharded(engines, group, ...)` drives the protocol for the engines this
process holds: all ranks in one process (LocalGroup: virtual ranks on one GPU,
or one process driving several GPUs) or one rank per process (DistGroup over
torch.distributed, NCCL between GPUs).
"""
import ctypes

import numpy as np

from ctypes import byref, c_double, c_int32, c_int64

from . import _lib
from ._lib import PPEvolveOpts, check, lib
from .errors import ArgumentError
from .paulis import pack_word, qubit_mask
from .truncation import NoTruncation, compile_filter, is_compilable


def owners(nw, z, x, rank_bits):
    """Owner rank of each key (host-side): z, x are (n, nw) uint64 arrays."""
    z = np.ascontiguousarray(z, dtype=np.uint64).reshape(-1, nw)
    x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, nw)
    out = np.zeros(len(z), dtype=np.int32)
    check(lib.pp_shard_owner(nw, z.ctypes.data, x.ctypes.data, len(z), rank_bits, out.ctypes.data))
    return out


def split(nw, z, x, c, rank_bits):
    """The terms (z, x, c) split by owner: a list of 2^rank_bits (z, x, c) parts."""
    o = owners(nw, z, x, rank_bits)
    return [(z[o == r], x[o == r], c[o == r]) for r in range(1 << rank_bits)]


def bits_for(n, cap, load_div):
    """Bucket bits for n local terms at a mean load of at most cap / load_div."""
    b = 1
    while b < 26 and (cap << b) < load_div * n:
        b += 1
    return b


class GpuShard:
    """One rank's engine: a SparsePauliVector holding the keys this rank owns."""

    def __init__(self, v, rank_bits, rank):
        import torch
        self.v, self.rank_bits, self.rank = v, rank_bits, rank
        self.torch = torch
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.nw = v.nw
        self._buf = None

    def tuning(self):
        from . import tune
        return tune.get_tuning(self.v)

    def local_terms(self):
        return len(self.v)

    def begin(self, gz, gx, cosv, sinv, opts, bits):
        mx = c_int32(0)
        check(lib.pp_shard_begin(self.v._h, self.rank_bits, self.rank, gz.ctypes.data, gx.ctypes.data,
                                 cosv.ctypes.data, sinv.ctypes.data, len(cosv), byref(opts), bits, byref(mx)))
        return mx.value

    def _buffers(self, cap):
        t = self.torch
        if self._buf is None or self._buf[2].numel() < cap:
            cap = max(cap, 1024)
            self._buf = (t.empty((cap, self.nw), dtype=t.int64, device=self.dev),
                         t.empty((cap, self.nw), dtype=t.int64, device=self.dev),
                         t.empty(cap, dtype=t.float64, device=self.dev))
        return self._buf

    def send(self, r, pref):
        """(partner, payload): payload = (z, x, c) device tensors of the terms to send."""
        cap = max(1, self.local_terms_now)
        z, x, c = self._buffers(cap)
        n, partner = c_int64(0), c_int32(0)
        check(lib.pp_shard_send(self.v._h, r, 1 if pref else 0, z.data_ptr(), x.data_ptr(), c.data_ptr(),
                                c.numel(), byref(n), byref(partner)))
        m = n.value
        return partner.value, (z[:m], x[:m], c[:m])

    def empty_payload(self, n):
        t = self.torch
        return (t.empty((n, self.nw), dtype=t.int64, device=self.dev),
                t.empty((n, self.nw), dtype=t.int64, device=self.dev),
                t.empty(n, dtype=t.float64, device=self.dev))

    def recv(self, payload):
        z, x, c = payload
        n = c.numel()
        if n:
            z, x, c = z.contiguous(), x.contiguous(), c.contiguous()
            check(lib.pp_shard_recv(self.v._h, z.data_ptr(), x.data_ptr(), c.data_ptr(), n))

    def rotate(self, r, pref):
        st = np.zeros(5, dtype=np.int64)
        check(lib.pp_shard_rotate(self.v._h, r, 1 if pref else 0, st.ctypes.data))
        self.local_terms_now = int(st[1])
        return [int(q) for q in st]

    def regrid(self, bits):
        mx = c_int32(0)
        check(lib.pp_shard_regrid(self.v._h, bits, byref(mx)))
        return mx.value

    def end(self):
        ev = c_double(0.0)
        st = np.zeros(_lib.PP_STATS_LEN, dtype=np.float64)
        check(lib.pp_shard_end(self.v._h, byref(ev), st.ctypes.data))
        return ev.value, {name: float(st[i]) for name, i in _lib.STAT.items()}


def _settle(payloads):
    """The copies into received payloads (made on torch's current stream of each
    payload's device) are complete before an engine's own stream reads them."""
    devices = {p[2].device for p in payloads if p is not None and p[2].is_cuda}
    if devices:
        import torch
        for d in devices:
            torch.cuda.current_stream(d).synchronize()


class LocalGroup:
    """Every rank in this process: exchanges are copies between the engines."""

    def __init__(self, size):
        self.size = size

    def exchange(self, engines, sends):
        by_rank = {e.rank: (p, pay) for e, (p, pay) in zip(engines, sends)}
        out = []
        for e, (partner, _) in zip(engines, sends):
            if partner == e.rank:
                out.append(None)
            else:
                p2, pay = by_rank[partner]
                assert p2 == e.rank, "partner ranks must pair up"
                dev = getattr(e, "dev", None)     # the receiving rank's device (engines on several GPUs)
                out.append(tuple(t.clone() if dev is None else t.to(dev, copy=True) for t in pay))
        _settle(out)
        return out

    def allreduce(self, values, op):
        return sum(values) if op == "sum" else max(values)


class DistGroup:
    """One rank per process over torch.distributed (NCCL between GPUs, gloo on CPU)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.size = dist.get_world_size(group)

    def exchange(self, engines, sends):
        (e,), ((partner, pay),) = engines, sends
        if partner == e.rank:
            return [None]
        t = e.torch
        dev = pay[2].device
        n_out = t.tensor([pay[2].numel()], dtype=t.int64, device=dev)
        n_in = t.zeros(1, dtype=t.int64, device=dev)
        self._swap([n_out], [n_in], partner)
        recv = e.empty_payload(int(n_in.item()))
        self._swap([q.contiguous() for q in pay], list(recv), partner)
        _settle([recv])
        return [recv]

    def _swap(self, outs, ins, partner):
        dist = self.dist
        ops = [dist.P2POp(dist.isend, o, partner, self.group) for o in outs if o.numel()]
        ops += [dist.P2POp(dist.irecv, i, partner, self.group) for i in ins if i.numel()]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce(self, values, op):
        import torch
        (v,) = values
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM if op == "sum" else self.dist.ReduceOp.MAX,
                             group=self.group)
        return t.item()


def _gen_arrays(N, generators, angles):
    """Generator key words and libm cos / sin of the angles, prepared as evolve_ does."""
    from .spv import _cos_sin, _gen_words
    gz, gx = _gen_words(N, generators)
    cosv, sinv = _cos_sin(angles)
    return gz, gx, cosv, sinv


def run_sharded(engines, group, N, generators, angles, *, truncation=None, local_truncation=None, channel=None,
                channel_every=0, append_capacity, ket=0, load_div=6):
    """evolve!(v, generators, angles; truncation, local_truncation) at window 1 on a
    key-sharded vector, followed by `channel` after every `channel_every` rotations.

    engines: this process's ranks (GpuShard or an equivalent engine), each holding
    the terms it owns.  append_capacity: the unsharded vector's append capacity
    (its early-merge rule).  Returns (<ket|O|ket> over all ranks, stats)."""
    from .spv import CHANNEL_KINDS, _pp_filter
    if len(generators) != len(angles):
        raise ArgumentError("generators and angles must have same length")
    truncation = truncation or NoTruncation()
    local_truncation = local_truncation or NoTruncation()
    if not (is_compilable(truncation) and is_compilable(local_truncation)):
        raise NotImplementedError("key-sharded runs take compiled (coefficient / weight) truncations")
    L = len(generators)
    opts = PPEvolveOpts()
    opts.window = 1
    strict_f = _pp_filter(compile_filter(truncation))
    local_f = _pp_filter(compile_filter(local_truncation))
    opts.strict = ctypes.pointer(strict_f)
    opts.local = ctypes.pointer(local_f)
    opts.strict_kind = 0
    opts.chan_kind = -1
    ketw = pack_word(N, ket)
    opts.ket = ketw.ctypes.data
    mask_w = None
    if channel is not None:
        kind, prm, qubits = channel
        opts.chan_kind = CHANNEL_KINDS[kind]
        prm = list(prm) if isinstance(prm, (list, tuple)) else [float(prm)]
        for i, p in enumerate(prm[:3]):
            opts.chan_prm[i] = float(p)
        mask_w = pack_word(N, qubit_mask(N, qubits))
        opts.chan_mask = mask_w.ctypes.data
    opts.chan_every = int(channel_every or 0)
    gz, gx, cosv, sinv = _gen_arrays(N, generators, angles)
    caps = {e.tuning()[0] for e in engines}
    if len(caps) != 1:
        raise ArgumentError("every rank needs the same bucket capacity")
    cap = caps.pop()
    if group.allreduce([cap], "max") != cap:
        raise ArgumentError("every rank needs the same bucket capacity")
    local_n = [e.local_terms() for e in engines]
    for e, n in zip(engines, local_n):
        e.local_terms_now = n
    gn = group.allreduce([sum(local_n)], "sum")
    bits = bits_for(int(group.allreduce([max(local_n)], "max")), cap, load_div)
    mx = group.allreduce([max(e.begin(gz, gx, cosv, sinv, opts, bits) for e in engines)], "max")
    while mx > cap // 2:
        bits += 1
        mx = group.allreduce([max(e.regrid(bits) for e in engines)], "max")
    acap = int(append_capacity)
    peak = 0
    for r in range(L):
        pref = gn > acap
        sends = [e.send(r, pref) for e in engines]
        recvd = group.exchange(engines, sends)
        for e, p in zip(engines, recvd):
            if p is not None:
                e.recv(p)
        st = [e.rotate(r, pref) for e in engines]
        gn = group.allreduce([sum(q[1] for q in st)], "sum")
        peak = max(peak, gn)
        if pref:
            gnp = group.allreduce([sum(q[3] for q in st)], "sum")
            if gnp > acap:
                acap = max(2 * acap, int(gnp))
        mx = group.allreduce([max(q[4] for q in st)], "max")
        while r + 1 < L and mx > cap // 2:
            bits += 1
            mx = group.allreduce([max(e.regrid(bits) for e in engines)], "max")
    parts = [e.end() for e in engines]
    expect = group.allreduce([sum(p[0] for p in parts)], "sum")
    stats = {k: group.allreduce([sum(p[1].get(k, 0.0) for p in parts)], "sum")
             for k in ("terms_in", "created", "merge_in", "merge_out")}
    stats["peak"] = peak
    stats["append_capacity"] = acap
    stats["bucket_bits"] = bits
    return expect, stats
