"""pauliprop.shard's protocol over torch.distributed on CPU: two gloo ranks
(world size 2, one process each, rendezvous on 127.0.0.1) run run_sharded with
DistGroup -- the pairwise exchange of sin-branch sources, the early-merge rule
from counts summed over ranks, the rank-ordered reductions -- with each rank's
engine a plain-Python restatement of one rank's rotation (test infrastructure:
the CUDA engine behind the same calls is tested on a GPU in test_gpu_shard.py).
The union of the two shards must equal the oracle's unsharded evolve!
(spv_evolve.jl:312-387) bit for bit."""
import multiprocessing as mp
import os
import random
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def popc(v):
    return bin(v).count("1")


class FakeShard:
    """One rank's terms in a dict, with the calls of pauliprop.shard.GpuShard."""

    def __init__(self, N, terms, rank_bits, rank, thresh, wmax):
        import torch
        self.torch, self.N, self.nw = torch, N, 1
        self.L, self.F = dict(terms), {}
        self.rank_bits, self.rank, self.thresh, self.wmax = rank_bits, rank, thresh, wmax

    def tuning(self):
        return (512, 4, 6, 128)

    def local_terms(self):
        return len(self.L)

    def begin(self, gz, gx, cosv, sinv, opts, bits):
        self.G = [(int(gz[i, 0]), int(gx[i, 0])) for i in range(len(cosv))]
        self.cos, self.sin = [float(a) for a in cosv], [float(a) for a in sinv]
        return 0

    def regrid(self, bits):
        return 0

    def drop(self, k, c):
        return abs(c) <= self.thresh or popc(k[0] | k[1]) > self.wmax

    @staticmethod
    def phase(k, M):
        (pz, px), (gz, gx) = k, M
        m1, m2 = popc(gx & pz), popc(gz & px)
        if (m1 - m2) & 1 == 0:
            return False, None, 0.0
        qz, qx = gz ^ pz, gx ^ px
        kk = (popc(qz & qx) - popc(gz & gx) - popc(pz & px) + 2 * m1) & 3
        return True, (qz, qx), float(kk - 2)

    def partner(self, r):
        import numpy as np
        from pauliprop import shard
        gz, gx = self.G[r]
        o = shard.owners(1, np.array([[gz]], dtype=np.uint64), np.array([[gx]], dtype=np.uint64), self.rank_bits)
        return self.rank ^ int(o[0])

    def _tensors(self, items):
        import numpy as np
        t = self.torch
        z = np.array([[k[0]] for k, _ in items], dtype=np.uint64).reshape(-1, 1).view(np.int64)
        x = np.array([[k[1]] for k, _ in items], dtype=np.uint64).reshape(-1, 1).view(np.int64)
        c = np.array([c for _, c in items], dtype=np.float64)
        return t.from_numpy(z.copy()), t.from_numpy(x.copy()), t.from_numpy(c)

    def send(self, r, pref):
        p = self.partner(r)
        items = []
        if p != self.rank:
            for k, c in self.L.items():
                if not (pref and self.drop(k, c)) and self.phase(k, self.G[r])[0]:
                    items.append((k, c))
        return p, self._tensors(items)

    def empty_payload(self, n):
        t = self.torch
        return t.empty((n, 1), dtype=t.int64), t.empty((n, 1), dtype=t.int64), t.empty(n, dtype=t.float64)

    def recv(self, payload):
        import numpy as np
        z, x, c = (q.numpy() for q in payload)
        z, x = z.view(np.uint64).reshape(-1), x.view(np.uint64).reshape(-1)
        self.F = {(int(z[i]), int(x[i])): float(c[i]) for i in range(len(c))}

    def rotate(self, r, pref):
        M, cv, sv = self.G[r], self.cos[r], self.sin[r]
        remote = self.partner(r) != self.rank
        n_in = len(self.L)
        live = {k: c for k, c in self.L.items() if not (pref and self.drop(k, c))}
        out, created = {}, 0
        for k, c in live.items():
            anti, q, sg = self.phase(k, M)
            v = c
            if anti:
                v = c * cv
                s = (sg * sv) * c
                created += 1
                src = self.F if remote else live
                if q in src:
                    v = v + (-(sg * sv)) * src[q]      # live value first, then the partner's sin branch
                elif not remote and not self.drop(q, s):
                    out[q] = s
            if not self.drop(k, v):
                out[k] = v
        if remote:
            for qk, cq in self.F.items():
                _, k, sg = self.phase(qk, M)
                if k not in live:
                    s = (sg * sv) * cq
                    if not self.drop(k, s):
                        out[k] = s
        self.F, self.L = {}, out
        return [n_in, len(out), created, len(live), 0]

    def end(self):
        e = sum(c for k, c in sorted(self.L.items()) if k[1] == 0)
        return e, {"terms_in": 0.0, "created": 0.0, "merge_in": 0.0, "merge_out": 0.0}


def _case(seed, n_terms=3000, L=30, N=40):
    rng = random.Random(seed)
    terms = {}
    while len(terms) < n_terms:
        z, x = rng.getrandbits(N), rng.getrandbits(N)
        for q in range(N):                  # mostly low weight
            if rng.random() < 0.8:
                z &= ~(1 << q)
                x &= ~(1 << q)
        terms[(z, x)] = rng.uniform(-1.0, 1.0)
    gens, angs = [], []
    for _ in range(L):
        a, b = rng.sample(range(N), 2)
        gens.append(((1 << a) | (1 << b), 0) if rng.random() < 0.5 else (0, 1 << a))
        angs.append(rng.uniform(0.2, 1.2))
    return terms, gens, angs


def _worker(rank, ws, port, q, seed, acap):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "paulioperators.jl_b200")]
    try:
        import datetime

        import numpy as np
        import torch.distributed as dist
        from pauliprop import shard
        from pauliprop.truncation import CoeffTruncation, CompositeTruncation, WeightTruncation
        dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
        terms, gens, angs = _case(seed)
        keys = list(terms)
        z = np.array([[k[0]] for k in keys], dtype=np.uint64)
        x = np.array([[k[1]] for k in keys], dtype=np.uint64)
        own = shard.owners(1, z, x, 1)
        mine = {k: terms[k] for k, o in zip(keys, own) if o == rank}
        eng = FakeShard(40, mine, 1, rank, 1e-2, 12)
        strat = CompositeTruncation(CoeffTruncation(1e-2), WeightTruncation(12))
        e, st = shard.run_sharded([eng], shard.DistGroup(), 40, gens, angs, truncation=strat, append_capacity=acap)
        q.put((rank, eng.L, e, st))
        dist.destroy_process_group()
    except Exception as ex:   # report instead of hanging the parent
        import traceback
        q.put(("error", traceback.format_exc(), repr(ex), None))


def _oracle_terms(seed, acap):
    sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import orc
    from helpers import filt
    terms, gens, angs = _case(seed)
    v = orc.OracleSPV(40, max(16, 2 * len(terms)), acap)
    v.upload([k[0] for k in terms], [k[1] for k in terms], list(terms.values()))
    v.evolve(gens, angs, window=1, strict=filt(("comp", [("coeff", 1e-2), ("weight", 12)])))
    oz, ox, oc = v.arrays()
    ref = {(int(oz[i, 0]), int(ox[i, 0])): float(oc[i]) for i in range(len(oc))}
    diag = ox[:, 0] == 0
    return ref, v.expect(0), float(abs(oc[diag]).sum())


@pytest.mark.parametrize("acap", [1 << 20, 40])
def test_sharded_protocol_local_group(acap):
    """The same protocol with both ranks in this process (LocalGroup: the
    exchange is a copy between the engines, as for virtual ranks on one GPU)."""
    sys.path[:0] = [ROOT, os.path.join(ROOT, "paulioperators.jl_b200")]
    import numpy as np
    from pauliprop import shard
    from pauliprop.truncation import CoeffTruncation, CompositeTruncation, WeightTruncation
    seed = 21
    terms, gens, angs = _case(seed)
    keys = list(terms)
    z = np.array([[k[0]] for k in keys], dtype=np.uint64)
    x = np.array([[k[1]] for k in keys], dtype=np.uint64)
    own = shard.owners(1, z, x, 1)
    engines = [FakeShard(40, {k: terms[k] for k, o in zip(keys, own) if o == r}, 1, r, 1e-2, 12) for r in range(2)]
    strat = CompositeTruncation(CoeffTruncation(1e-2), WeightTruncation(12))
    e, st = shard.run_sharded(engines, shard.LocalGroup(2), 40, gens, angs, truncation=strat, append_capacity=acap)
    union = {}
    for eng in engines:
        assert not (set(eng.L) & set(union))
        union.update(eng.L)
    ref, ev, scale = _oracle_terms(seed, acap)
    assert len(union) == len(ref) > 0 and set(union) == set(ref), "key sets differ"
    assert all(union[k] == ref[k] for k in ref), "coefficients differ"
    assert abs(e - ev) <= 1e-12 * max(1e-300, scale)
    if acap == 40:
        assert st["append_capacity"] > 40


@pytest.mark.parametrize("acap", [1 << 20, 40])
def test_sharded_protocol_two_gloo_ranks(acap):
    """acap 2^20: no early merge; acap 40: the global count passes it, so the
    rotations pre-filter and the capacity grows from the summed survivors."""
    sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import orc
    from helpers import filt
    seed = 21
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, seed, acap)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=300) for _ in procs]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(r[0] != "error" for r in res), [r[1] for r in res if r[0] == "error"]
    union = {}
    for _, part, _, _ in res:
        assert not (set(part) & set(union))
        union.update(part)
    terms, gens, angs = _case(seed)
    v = orc.OracleSPV(40, max(16, 2 * len(terms)), acap)
    v.upload([k[0] for k in terms], [k[1] for k in terms], list(terms.values()))
    v.evolve(gens, angs, window=1, strict=filt(("comp", [("coeff", 1e-2), ("weight", 12)])))
    oz, ox, oc = v.arrays()
    ref = {(int(oz[i, 0]), int(ox[i, 0])): float(oc[i]) for i in range(len(oc))}
    assert len(union) == len(ref) > 0
    assert set(union) == set(ref), "key sets differ"
    assert all(union[k] == ref[k] for k in ref), "coefficients differ"
    diag = ox[:, 0] == 0
    assert abs(res[0][2] - v.expect(0)) <= 1e-12 * max(1e-300, float(abs(oc[diag]).sum()))
    assert res[0][3]["append_capacity"] == res[1][3]["append_capacity"]
    if acap == 40:
        assert res[0][3]["append_capacity"] > 40
