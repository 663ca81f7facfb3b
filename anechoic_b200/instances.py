"""Ising / Max-Cut instances: integer couplings J (int8, symmetric, zero diagonal) and an optional integer bias.

File formats (same byte layout as the reference's loaders, gpu/multibit_bias_20261008/src/jmat.hpp:1-10 and
gpu/onsager_v2_20261007/src/sca_ref.hpp:23-49):

* SNOWGPU1 -- 8-byte magic, uint32 N, then N rows of 32 little-endian uint64 words (2048 bits); bit y of row x is 1 iff
  J_xy = +1 (a +-1 complete graph; N = 2000 in the reference).
* SCAJINT8 -- 8-byte magic, uint32 N, uint32 0, then N*N int8 row-major.
* SCABIAS1 -- 8-byte magic, uint32 N, uint32 0, then N int32 biases (|b| <= 32767).
* G-set text -- "n m" then m lines "i j w" (1-based); J = -w.

Generators are pure functions of their seed (splitmix64 streams), so an instance is named by its parameters:

* ``random_kbit`` follows the stream of the reference generator ``gen_ising random``
  (gpu/multibit_bias_20261008/src/gen_ising.cpp:118-143): per pair x < y (row-major) two draws r0, r1 from
  splitmix64(seed ^ 0xA5A5F00D12345678); J = 0 with probability pzero (r0 < pzero * 2^64), else |J| = 1 + (r1 >> 1) % M,
  negative iff r1 & 1; biases uniform in [-bmax, bmax] from splitmix64(seed ^ 0x5B1A5B1A5B1A5B1A). It is generalised here
  to any N (the reference caps N at 2048).
* ``complete_pm1`` is ``random_kbit(n, K=2, pzero=0)``: iid uniform +-1 couplings on the complete graph.
* Sparse classes shaped like the reference's G-set study (research/gset_20261007/synth.py:15-31): uniform random graphs
  with m edges, 2-D toroidal grids, +1 or iid +-1 weights. These are synthetic stand-ins, never G-set files.
"""
from __future__ import annotations

import dataclasses
import math
import struct
from typing import Optional

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def pad_spins(n: int) -> int:
    """Padded spin count NP(n) = max(2048, ceil(n / 256) * 256): 256 RNG lanes, NP / 256 rounds per step."""
    return max(2048, -(-n // 256) * 256)


def spin_words(n: int) -> int:
    """uint64 words per spin vector (32 for n <= 2048, as the reference's spins.bin records)."""
    return pad_spins(n) // 64


def splitmix64_block(state: int, start: int, count: int) -> np.ndarray:
    """Outputs start .. start+count-1 (0-based) of the splitmix64 stream seeded with `state`."""
    k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(state) + k * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


@dataclasses.dataclass
class Instance:
    """Couplings as dense int8 (n x n) or CSR rows, plus an optional bias. Derived quantities follow jmat::finish
    (gpu/multibit_bias_20261008/src/jmat.hpp:21-40)."""

    n: int
    dense: Optional[np.ndarray] = None          # int8 [n, n]
    row_ptr: Optional[np.ndarray] = None        # int32 [n + 1]
    col: Optional[np.ndarray] = None            # int32 [nnz]
    val: Optional[np.ndarray] = None            # int8 [nnz]
    bias: Optional[np.ndarray] = None           # int32 [n]
    name: str = ""

    def __post_init__(self):
        if (self.dense is None) == (self.row_ptr is None):
            raise ValueError("give exactly one of dense / CSR couplings")
        if self.dense is not None:
            self.dense = np.ascontiguousarray(self.dense, np.int8)
            if self.dense.shape != (self.n, self.n):
                raise ValueError("dense J must be n x n")
        else:
            self.row_ptr = np.ascontiguousarray(self.row_ptr, np.int32)
            self.col = np.ascontiguousarray(self.col, np.int32)
            self.val = np.ascontiguousarray(self.val, np.int8)
        if self.bias is not None:
            self.bias = np.ascontiguousarray(self.bias, np.int32)
            if self.bias.shape != (self.n,):
                raise ValueError("bias must have n entries")

    @property
    def is_sparse(self) -> bool:
        return self.dense is None

    def to_csr(self):
        if self.is_sparse:
            return self.row_ptr, self.col, self.val
        nz = self.dense != 0
        counts = nz.sum(axis=1)
        rp = np.zeros(self.n + 1, np.int32)
        rp[1:] = np.cumsum(counts)
        ys = np.nonzero(nz)
        return rp, ys[1].astype(np.int32), self.dense[ys].astype(np.int8)

    def to_dense(self) -> np.ndarray:
        if not self.is_sparse:
            return self.dense
        d = np.zeros((self.n, self.n), np.int8)
        rows = np.repeat(np.arange(self.n), np.diff(self.row_ptr))
        d[rows, self.col] = self.val
        return d

    # ---- derived quantities (jmat::finish) ----
    def stats(self) -> dict:
        rp, col, val = self.to_csr()
        v = val.astype(np.int64)
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        upper = col > rows
        sumw = -int(v[upper].sum())
        rowabs = np.zeros(self.n, np.int64)
        np.add.at(rowabs, rows, np.abs(v))
        maxabs = int(np.abs(v).max()) if len(v) else 0
        bmax = int(np.abs(self.bias).max()) if self.bias is not None and self.n else 0
        return dict(n=self.n, nnz=int(len(v)), sumw=sumw, maxabs=maxabs, hmax=int(rowabs.max()) if self.n else 0,
                    bmax=bmax, mean_row_sq=float((v * v).sum()) / self.n)

    def kbits(self) -> int:
        """Smallest K in {1, 2, 4, 8} whose planes hold J (K = 1 only for a +-1 complete graph)."""
        st = self.stats()
        if st["nnz"] == self.n * (self.n - 1) and st["maxabs"] == 1:
            return 1
        for K in (2, 4, 8):
            if st["maxabs"] <= (1 << (K - 1)) - 1:
                return K
        raise ValueError("|J| > 127")

    def validate(self):
        """Symmetric, zero diagonal (jmat::finish's checks)."""
        if self.is_sparse:
            d = self.to_dense() if self.n <= 4096 else None
            rows = np.repeat(np.arange(self.n), np.diff(self.row_ptr))
            if np.any(self.col == rows):
                raise ValueError("nonzero diagonal coupling")
            key = rows.astype(np.int64) * self.n + self.col
            keyT = self.col.astype(np.int64) * self.n + rows
            o1, o2 = np.argsort(key), np.argsort(keyT)
            if not (np.array_equal(key[o1], keyT[o2]) and np.array_equal(self.val[o1], self.val[o2])):
                raise ValueError("J not symmetric")
            del d
        else:
            if np.any(np.diagonal(self.dense) != 0):
                raise ValueError("nonzero diagonal coupling")
            if not np.array_equal(self.dense, self.dense.T):
                raise ValueError("J not symmetric")
        if self.bias is not None and np.any(np.abs(self.bias.astype(np.int64)) > 32767):
            raise ValueError("bias outside |b| <= 32767")

    # ---- independent scorers (jmat.hpp:130-161) ----
    def spins_pm(self, bits: np.ndarray) -> np.ndarray:
        b = np.asarray(bits, np.uint64)
        i = np.arange(self.n)
        up = (b[i >> 6] >> (i & 63).astype(np.uint64)) & np.uint64(1)
        return np.where(up == 1, 1, -1).astype(np.int64)

    def cut(self, bits) -> int:
        """Max-Cut value sum_{x<y, s_x != s_y} w_xy with w = -J."""
        s = self.spins_pm(bits)
        rp, col, val = self.to_csr()
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        m = (col > rows) & (s[rows] != s[col])
        return int(-val[m].astype(np.int64).sum())

    def energy(self, bits) -> int:
        """E = -sum_{x<y} J_xy s_x s_y - sum_x b_x s_x."""
        s = self.spins_pm(bits)
        rp, col, val = self.to_csr()
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        m = col > rows
        e = -int((val[m].astype(np.int64) * s[rows[m]] * s[col[m]]).sum())
        if self.bias is not None:
            e -= int((self.bias.astype(np.int64) * s).sum())
        return e

    def fields(self, bits) -> np.ndarray:
        """h = b + J s recomputed from scratch (jmat::field_mismatches)."""
        s = self.spins_pm(bits)
        rp, col, val = self.to_csr()
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        h = np.zeros(self.n, np.int64)
        np.add.at(h, rows, val.astype(np.int64) * s[col])
        if self.bias is not None:
            h += self.bias
        return h


# ------------------------------------------------------------------------------------------------ generators
def random_kbit(n: int, K: int, seed: int, pzero: float = 0.0, bmax: int = 0, name: str = "") -> Instance:
    """Dense random K-bit couplings and bias with the stream of gen_ising random (gen_ising.cpp:118-143)."""
    if K < 2 or K > 8 or n < 1:
        raise ValueError("2 <= K <= 8, n >= 1")
    M = (1 << (K - 1)) - 1
    st = (seed ^ 0xA5A5F00D12345678) & 0xFFFFFFFFFFFFFFFF
    lim = math.ldexp(pzero, 64)
    zthr = np.uint64(0xFFFFFFFFFFFFFFFF) if lim >= 18446744073709551615.0 else np.uint64(int(lim))
    J = np.zeros((n, n), np.int8)
    pos = 0
    for x in range(n - 1):
        cnt = n - 1 - x
        z = splitmix64_block(st, 2 * pos, 2 * cnt)
        r0, r1 = z[0::2], z[1::2]
        mag = (1 + ((r1 >> np.uint64(1)) % np.uint64(M))).astype(np.int16)
        v = np.where((r1 & np.uint64(1)) == 1, -mag, mag)
        if pzero > 0:
            v = np.where(r0 < zthr, 0, v)
        J[x, x + 1:] = v
        pos += cnt
    J = J + J.T
    bias = None
    if bmax > 0:
        sb = (seed ^ 0x5B1A5B1A5B1A5B1A) & 0xFFFFFFFFFFFFFFFF
        z = splitmix64_block(sb, 0, n)
        bias = ((z % np.uint64(2 * bmax + 1)).astype(np.int64) - bmax).astype(np.int32)
    return Instance(n=n, dense=J, bias=bias, name=name or f"rand_k{K}_n{n}_s{seed}")


def complete_pm1(n: int, seed: int) -> Instance:
    """Complete graph, J_xy = J_yx iid uniform in {-1, +1}, zero diagonal (random_kbit with K = 2, pzero = 0)."""
    inst = random_kbit(n, 2, seed)
    inst.name = f"complete_pm1_n{n}_s{seed}"
    return inst


def _from_edges(n, i, j, w, bias, name) -> Instance:
    """Sparse instance from an edge list (i < j, Max-Cut weights w, J = -w)."""
    i = np.asarray(i, np.int64); j = np.asarray(j, np.int64); Jv = (-np.asarray(w, np.int64)).astype(np.int8)
    rows = np.concatenate([i, j]); cols = np.concatenate([j, i]); vals = np.concatenate([Jv, Jv])
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    return Instance(n=n, row_ptr=rp, col=cols.astype(np.int32), val=vals, bias=bias, name=name)


def _weights(rng, m, signed):
    return rng.choice(np.array([-1, 1]), size=m) if signed else np.ones(m, np.int64)


def _bias(n, bmax, seed):
    if bmax <= 0:
        return None
    z = splitmix64_block((seed ^ 0x5B1A5B1A5B1A5B1A) & 0xFFFFFFFFFFFFFFFF, 0, n)
    return ((z % np.uint64(2 * bmax + 1)).astype(np.int64) - bmax).astype(np.int32)


def random_graph(n: int, m: int, signed: bool, seed: int, bmax: int = 0) -> Instance:
    """Uniform random graph with m distinct edges, weights +1 or iid +-1."""
    rng = np.random.default_rng(seed)
    total = n * (n - 1) // 2
    pick = np.sort(rng.choice(total, size=m, replace=False))
    # unrank pair index -> (i, j), i < j, row-major over the upper triangle
    i = np.zeros(m, np.int64)
    starts = np.concatenate([[0], np.cumsum(np.arange(n - 1, 0, -1))])
    i = np.searchsorted(starts, pick, side="right") - 1
    j = pick - starts[i] + i + 1
    return _from_edges(n, i, j, _weights(rng, m, signed), _bias(n, bmax, seed),
                       f"rand_n{n}_m{m}_{'pm' if signed else 'p'}_s{seed}")


def torus(L1: int, L2: int, seed: int, signed: bool = True, bmax: int = 0) -> Instance:
    """2-D toroidal grid L1 x L2 (each vertex joined to its right and lower neighbour), weights +1 or iid +-1."""
    rng = np.random.default_rng(seed)
    idx = np.arange(L1 * L2).reshape(L1, L2)
    a = np.concatenate([idx.ravel(), idx.ravel()])
    b = np.concatenate([np.roll(idx, -1, 0).ravel(), np.roll(idx, -1, 1).ravel()])
    i, j = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(i * (L1 * L2) + j)
    i, j = key // (L1 * L2), key % (L1 * L2)
    n = L1 * L2
    return _from_edges(n, i, j, _weights(rng, len(i), signed), _bias(n, bmax, seed),
                       f"torus_{L1}x{L2}_{'pm' if signed else 'p'}_s{seed}")


def sparse_classes_manifest(seed: int = 20261008, bmax: int = 2):
    """51 synthetic sparse instances of uneven size shaped like the G-set classes (uniform random graphs with the
    classes' sizes and edge counts, +1 or +-1 weights, and toroidal grids from N = 800 up to N = 20000), each with an
    integer bias uniform in [-bmax, bmax]. Returns a list of (name, builder) pairs; builders are pure functions."""
    spec = []
    for c in range(5):
        spec.append(("R800p", lambda s, c=c: random_graph(800, 19176, False, s + c, bmax)))
    for c in range(5):
        spec.append(("R800pm", lambda s, c=c: random_graph(800, 19176, True, s + c, bmax)))
    for c in range(8):   # degree ~12 (planar-like classes' edge density): 800 / 1000 / 2000 vertices
        nn, mm = [(800, 4690), (800, 4670), (1000, 5910), (1000, 5915), (2000, 11778), (2000, 11770),
                  (2000, 11785), (2000, 11779)][c]
        spec.append((f"D{nn}", lambda s, c=c, nn=nn, mm=mm: random_graph(nn, mm, c % 2 == 1, s + 100 + c, bmax)))
    for c in range(10):
        spec.append(("R2000", lambda s, c=c: random_graph(2000, 19990, c >= 5, s + 200 + c, bmax)))
    for c in range(5):
        spec.append(("R1000p", lambda s, c=c: random_graph(1000, 9990, False, s + 300 + c, bmax)))
    for c in range(10):
        spec.append(("D6", lambda s, c=c: random_graph(1000 + 500 * c, 3 * (1000 + 500 * c), c % 2 == 0,
                                                       s + 400 + c, bmax)))
    for L1, L2 in [(20, 40), (20, 40), (20, 40), (40, 50), (40, 50), (50, 60), (70, 100), (100, 100)]:
        spec.append((f"T{L1 * L2}", lambda s, L1=L1, L2=L2: torus(L1, L2, s + L1 * 1000 + L2, True, bmax)))
    assert len(spec) == 51
    spec[-1] = ("T20000", lambda s: torus(100, 200, s + 100200, True, bmax))
    return [(f"{cls}_{k}", (lambda b=b: b(seed))) for k, (cls, b) in enumerate(spec)]


# ------------------------------------------------------------------------------------------------ file formats
def read_snowgpu1(path: str) -> Instance:
    with open(path, "rb") as f:
        magic = f.read(8)
        if magic != b"SNOWGPU1":
            raise ValueError("bad graph header")
        (n,) = struct.unpack("<I", f.read(4))
        if n < 1 or n > 2048:
            raise ValueError("bad graph header")
        words = np.frombuffer(f.read(8 * 32 * n), dtype="<u8")
        if words.size != 32 * n:
            raise ValueError("short graph file")
    bits = np.unpackbits(words.reshape(n, 32).view(np.uint8), axis=1, bitorder="little")[:, :n]
    J = np.where(bits == 1, 1, -1).astype(np.int8)
    np.fill_diagonal(J, 0)
    return Instance(n=n, dense=J, name=path)


def write_snowgpu1(inst: Instance, path: str):
    J = inst.to_dense()
    n = inst.n
    if n > 2048:
        raise ValueError("SNOWGPU1 holds n <= 2048")
    bits = np.zeros((n, 2048), np.uint8)
    bits[:, :n] = (J == 1)
    words = np.packbits(bits, axis=1, bitorder="little").view("<u8")
    with open(path, "wb") as f:
        f.write(b"SNOWGPU1"); f.write(struct.pack("<I", n)); f.write(words.tobytes())


def read_jint8(path: str) -> Instance:
    with open(path, "rb") as f:
        magic = f.read(8)
        n, rsv = struct.unpack("<II", f.read(8))
        if magic != b"SCAJINT8" or n < 1 or rsv != 0:
            raise ValueError("bad JINT8 header")
        data = f.read()
    if len(data) != n * n:
        raise ValueError("short or trailing JINT8 data")
    inst = Instance(n=n, dense=np.frombuffer(data, np.int8).reshape(n, n).copy(), name=path)
    inst.validate()
    return inst


def write_jint8(inst: Instance, path: str):
    with open(path, "wb") as f:
        f.write(b"SCAJINT8"); f.write(struct.pack("<II", inst.n, 0)); f.write(inst.to_dense().tobytes())


def read_bias(path: str, n: int) -> np.ndarray:
    with open(path, "rb") as f:
        magic = f.read(8)
        m, rsv = struct.unpack("<II", f.read(8))
        if magic != b"SCABIAS1" or rsv != 0:
            raise ValueError("bad bias header")
        if m != n:
            raise ValueError("bias length differs from N")
        data = f.read()
    if len(data) != 4 * n:
        raise ValueError("short or trailing bias data")
    b = np.frombuffer(data, "<i4").astype(np.int32)
    if np.any(np.abs(b.astype(np.int64)) > 32767):
        raise ValueError("bias outside |b| <= 32767 (B_BITS = 16)")
    return b


def write_bias(b: np.ndarray, path: str):
    b = np.asarray(b, np.int32)
    with open(path, "wb") as f:
        f.write(b"SCABIAS1"); f.write(struct.pack("<II", len(b), 0)); f.write(b.astype("<i4").tobytes())


def read_gset(path: str) -> Instance:
    with open(path) as f:
        tok = f.read().split()
    n, e = int(tok[0]), int(tok[1])
    arr = np.array(tok[2:2 + 3 * e], np.int64).reshape(e, 3)
    if len(tok) != 2 + 3 * e:
        raise ValueError("short or trailing G-set data")
    i, j, w = arr[:, 0] - 1, arr[:, 1] - 1, arr[:, 2]
    if np.any((i < 0) | (j < 0) | (i >= n) | (j >= n) | (i == j)):
        raise ValueError("bad G-set edge")
    if np.any(np.abs(w) > 127):
        raise ValueError("G-set weight out of int8 range")
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    if len(np.unique(lo * n + hi)) != e:
        raise ValueError("duplicate G-set edge")
    return _from_edges(n, lo, hi, w, None, path)


def write_gset(inst: Instance, path: str):
    rp, col, val = inst.to_csr()
    rows = np.repeat(np.arange(inst.n), np.diff(rp))
    m = col > rows
    with open(path, "w") as f:
        f.write(f"{inst.n} {int(m.sum())}\n")
        for a, b, v in zip(rows[m], col[m], val[m]):
            f.write(f"{a + 1} {b + 1} {-int(v)}\n")


def load(kind: str, path: str) -> Instance:
    """Load by explicit kind, as jmat::load (jmat.hpp:115-120): graph (SNOWGPU1), gset (edge list), jint8 (dense)."""
    if kind == "graph":
        return read_snowgpu1(path)
    if kind == "gset":
        return read_gset(path)
    if kind == "jint8":
        return read_jint8(path)
    raise ValueError("unknown J source kind " + kind)


def main(argv=None) -> int:
    """Write the synthetic instances of the benchmarks and tests as files the CLI reads:

        python -m anechoic_b200.instances complete --n 2000 --seed 20261004 --out F.bin        SNOWGPU1 (+-1 complete)
        python -m anechoic_b200.instances kbit --n 16384 --kbits 4 --seed S [--pzero P] [--bmax B] --out PREFIX
                                                                           PREFIX.jint8 (+ PREFIX.bias when B > 0)
        python -m anechoic_b200.instances torus --l1 100 --l2 200 --seed S [--plus] [--bmax B] --out PREFIX
                                                                           PREFIX.gset (+ PREFIX.bias when B > 0)
    """
    import argparse
    ap = argparse.ArgumentParser(prog="python -m anechoic_b200.instances")
    ap.add_argument("kind", choices=["complete", "kbit", "torus"])
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--kbits", type=int, default=4)
    ap.add_argument("--seed", type=int, default=20261004)
    ap.add_argument("--pzero", type=float, default=0.0)
    ap.add_argument("--bmax", type=int, default=0)
    ap.add_argument("--l1", type=int, default=100)
    ap.add_argument("--l2", type=int, default=200)
    ap.add_argument("--plus", action="store_true", help="torus: weights +1 instead of iid +-1")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    if a.kind == "complete":
        write_snowgpu1(complete_pm1(a.n, a.seed), a.out)
        print(a.out)
        return 0
    inst = random_kbit(a.n, a.kbits, a.seed, pzero=a.pzero, bmax=a.bmax) if a.kind == "kbit" else \
        torus(a.l1, a.l2, a.seed, signed=not a.plus, bmax=a.bmax)
    path = a.out + (".jint8" if a.kind == "kbit" else ".gset")
    (write_jint8 if a.kind == "kbit" else write_gset)(inst, path)
    print(path)
    if inst.bias is not None:
        write_bias(inst.bias, a.out + ".bias")
        print(a.out + ".bias")
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
