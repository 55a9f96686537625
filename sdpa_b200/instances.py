"""Seeded synthetic SDP instances in SDPA format, and the .dat-s writer.

The instance families are the workloads this solver is measured on:

* MaxCut relaxation of an Erdos-Renyi graph G(n, p): one n x n block,
  c = 1_m, F0 = L/4 (L the weighted graph Laplacian), F_i = e_i e_i^T.  In
  SDPA's dual form this is  max (L/4).Y  s.t. Y_ii = 1, Y psd.
* Lovasz theta of G(n, p): one n x n block, m = 1 + |E|, c = (1, 0, ..., 0),
  F0 = J (all ones), F1 = I, one F_k = E_ij per edge (upper entry 1).
* Random strictly feasible SDP: a dense n-block plus an LP block; every A_i
  has floor(density * n(n+1)/2) upper-triangle N(0,1) entries at uniformly
  chosen positions plus one LP diagonal entry; b_i = Tr(A_i) so X0 = I is
  feasible, C = sum_i y0_i A_i + I with y0 ~ N(0,1) so Z0 = I is feasible
  (file F0 = -C, c = b).
* Batched MaxCut: per seed s, n ~ U{20..120}, p ~ U(0.05, 0.3), edge weights
  U(0, 1).  Warm-start sets use n ~ U{50..200}.
* Batched multi-block: per seed, 2..4 SDP blocks of order U{6..40} and an LP
  block, built like the random SDP (strictly feasible from X = Y = I).

Indices in an `Instance` are 1-based exactly as in a .dat-s file (block l,
row i <= column j; k = 0 is F0).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Instance:
    m: int
    blocks: list          # signed block sizes as in the file (negative = LP)
    c: np.ndarray         # (m,) float64
    k: np.ndarray         # (nnz,) int32, matrix index 0..m
    l: np.ndarray         # (nnz,) int32, 1-based block
    i: np.ndarray         # (nnz,) int32, 1-based row    (i <= j)
    j: np.ndarray         # (nnz,) int32, 1-based column
    v: np.ndarray         # (nnz,) float64
    name: str = ""

    def to_dats(self) -> str:
        """SDPA sparse format text (the reader is IO::read, sdpa_io.cpp:33-73, :473-540)."""
        out = [f'"{self.name or "sdpa_b200 instance"}"',
               f"{self.m} = mDIM", f"{len(self.blocks)} = nBLOCK",
               " ".join(str(int(b)) for b in self.blocks) + " = bLOCKsTRUCT",
               " ".join(repr(float(x)) for x in self.c)]
        order = np.lexsort((self.j, self.i, self.l, self.k))
        for q in order:
            out.append(f"{int(self.k[q])} {int(self.l[q])} {int(self.i[q])} {int(self.j[q])} "
                       f"{float(self.v[q])!r}")
        return "\n".join(out) + "\n"

    def write(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.to_dats())


def _gnp_edges(n: int, p: float, rng: np.random.Generator):
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.size) < p
    return iu[keep], ju[keep]


def maxcut_from_graph(n: int, ei: np.ndarray, ej: np.ndarray, w: np.ndarray, name: str = "") -> Instance:
    """MaxCut SDP relaxation of a weighted graph (edges 0-based, ei < ej)."""
    deg = np.zeros(n)
    np.add.at(deg, ei, w)
    np.add.at(deg, ej, w)
    # F0 = L/4: diagonal deg/4, off-diagonal -w/4 (upper triangle only)
    dk = np.zeros(n, np.int32)
    di = np.arange(1, n + 1, dtype=np.int32)
    ok = deg != 0.0
    k = [dk[ok], np.zeros(ei.size, np.int32), np.arange(1, n + 1, dtype=np.int32)]
    ii = [di[ok], (ei + 1).astype(np.int32), di]
    jj = [di[ok], (ej + 1).astype(np.int32), di]
    vv = [deg[ok] / 4.0, -w / 4.0, np.ones(n)]
    return Instance(m=n, blocks=[n], c=np.ones(n), k=np.concatenate(k),
                    l=np.ones(sum(a.size for a in k), np.int32), i=np.concatenate(ii),
                    j=np.concatenate(jj), v=np.concatenate(vv), name=name)


def maxcut(n: int = 100, p: float = 0.1, seed: int = 1, unit_weights: bool = True) -> Instance:
    """MaxCut of G(n, p) from `seed` (numpy default_rng)."""
    rng = np.random.default_rng(seed)
    ei, ej = _gnp_edges(n, p, rng)
    w = np.ones(ei.size) if unit_weights else rng.uniform(0.0, 1.0, ei.size)
    return maxcut_from_graph(n, ei, ej, w, name=f"maxcut G({n},{p}) seed {seed}")


def batch_maxcut_params(seed: int, nmin: int = 20, nmax: int = 120):
    """(n, p, rng) of one batched-MaxCut instance: n ~ U{nmin..nmax}, p ~ U(0.05, 0.3)."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(nmin, nmax + 1))
    p = float(rng.uniform(0.05, 0.3))
    return n, p, rng


def batch_maxcut_graph(seed: int, nmin: int = 20, nmax: int = 120):
    """The weighted graph (n, ei, ej, w) of one batched-MaxCut instance."""
    n, p, rng = batch_maxcut_params(seed, nmin, nmax)
    ei, ej = _gnp_edges(n, p, rng)
    w = rng.uniform(0.0, 1.0, ei.size)
    return n, ei, ej, w


def batch_maxcut(seed: int, nmin: int = 20, nmax: int = 120) -> Instance:
    n, ei, ej, w = batch_maxcut_graph(seed, nmin, nmax)
    return maxcut_from_graph(n, ei, ej, w, name=f"batched maxcut seed {seed}")


def lovasz_theta(n: int = 200, p: float = 0.5, seed: int = 1) -> Instance:
    """Lovasz theta SDP of G(n, p) from `seed`."""
    rng = np.random.default_rng(seed)
    ei, ej = _gnp_edges(n, p, rng)
    ne = ei.size
    m = 1 + ne
    iu, ju = np.triu_indices(n)
    k = np.concatenate([np.zeros(iu.size, np.int32), np.ones(n, np.int32),
                        np.arange(2, m + 1, dtype=np.int32)])
    ii = np.concatenate([iu + 1, np.arange(1, n + 1), ei + 1]).astype(np.int32)
    jj = np.concatenate([ju + 1, np.arange(1, n + 1), ej + 1]).astype(np.int32)
    v = np.concatenate([np.ones(iu.size), np.ones(n), np.ones(ne)])
    c = np.zeros(m)
    c[0] = 1.0
    return Instance(m=m, blocks=[n], c=c, k=k, l=np.ones(k.size, np.int32), i=ii, j=jj, v=v,
                    name=f"lovasz theta G({n},{p}) seed {seed}")


def random_sdp(m: int = 2000, n: int = 500, nlp: int = 50, density: float = 0.01,
               lp_per_constraint: int = 1, seed: int = 1) -> Instance:
    """Random strictly feasible SDP with blocks {n, -nlp} (see module doc)."""
    rng = np.random.default_rng(seed)
    ntri = n * (n + 1) // 2
    per = int(np.floor(density * ntri))
    iu, ju = np.triu_indices(n)
    ks, ls, is_, js, vs = [], [], [], [], []
    C = np.zeros((n, n))
    Clp = np.ones(nlp)
    C[np.diag_indices(n)] = 1.0
    y0 = rng.standard_normal(m)
    b = np.zeros(m)
    for a in range(m):
        pos = rng.choice(ntri, size=per, replace=False)
        val = rng.standard_normal(per)
        r, s = iu[pos], ju[pos]
        lpi = rng.choice(nlp, size=lp_per_constraint, replace=False)
        lpv = rng.standard_normal(lp_per_constraint)
        ks += [np.full(per + lp_per_constraint, a + 1, np.int32)]
        ls += [np.concatenate([np.ones(per, np.int32), np.full(lp_per_constraint, 2, np.int32)])]
        is_ += [np.concatenate([r + 1, lpi + 1]).astype(np.int32)]
        js += [np.concatenate([s + 1, lpi + 1]).astype(np.int32)]
        vs += [np.concatenate([val, lpv])]
        b[a] = val[r == s].sum() + lpv.sum()
        np.add.at(C, (r, s), y0[a] * val)
        off = r != s
        np.add.at(C, (s[off], r[off]), y0[a] * val[off])
        np.add.at(Clp, lpi, y0[a] * lpv)
    # file F0 = -C (upper triangle, dense) and the LP part
    ks.insert(0, np.zeros(ntri + nlp, np.int32))
    ls.insert(0, np.concatenate([np.ones(ntri, np.int32), np.full(nlp, 2, np.int32)]))
    is_.insert(0, np.concatenate([iu + 1, np.arange(1, nlp + 1)]).astype(np.int32))
    js.insert(0, np.concatenate([ju + 1, np.arange(1, nlp + 1)]).astype(np.int32))
    vs.insert(0, np.concatenate([-C[iu, ju], -Clp]))
    return Instance(m=m, blocks=[n, -nlp], c=b, k=np.concatenate(ks), l=np.concatenate(ls),
                    i=np.concatenate(is_), j=np.concatenate(js), v=np.concatenate(vs),
                    name=f"random sdp m={m} n={n} lp={nlp} seed {seed}")


def random_block_sdp(m: int, blocks: list, density: float = 0.1, lp_per_constraint: int = 1,
                     seed: int = 1, name: str = "", touch: list | None = None) -> Instance:
    """Random strictly feasible SDP with the given signed block structure
    (positive = SDP block, negative = LP block), built like `random_sdp`:
    every A_i has floor(density * k(k+1)/2) (at least one) N(0,1) upper
    entries in each SDP block of order k it touches (each block with
    probability 0.7, at least one block; or the SDP blocks listed in
    touch[i], indices into the SDP blocks) plus `lp_per_constraint` LP
    entries; b_i = Tr(A_i), C = sum_i y0_i A_i + I, file F0 = -C, c = b."""
    rng = np.random.default_rng(seed)
    sdp = [(l + 1, int(k)) for l, k in enumerate(blocks) if k > 0]
    lps = [(l + 1, -int(k)) for l, k in enumerate(blocks) if k < 0]
    Cs = {l: np.eye(k) for l, k in sdp}
    Cl = {l: np.ones(k) for l, k in lps}
    y0 = rng.standard_normal(m)
    b = np.zeros(m)
    ks, ls, is_, js, vs = [], [], [], [], []

    def add(a, l, r, c, v):
        ks.append(np.full(r.size, a, np.int32))
        ls.append(np.full(r.size, l, np.int32))
        is_.append((r + 1).astype(np.int32))
        js.append((c + 1).astype(np.int32))
        vs.append(v)

    for a in range(m):
        if touch is not None:
            tl = list(touch[a])
        else:
            tl = [t for t in range(len(sdp)) if rng.random() < 0.7] if sdp else []
            if sdp and not tl:
                tl = [int(rng.integers(len(sdp)))]
        for t in tl:
            l, k = sdp[t]
            iu, ju = np.triu_indices(k)
            per = max(1, int(np.floor(density * iu.size)))
            pos = rng.choice(iu.size, size=per, replace=False)
            val = rng.standard_normal(per)
            r, c = iu[pos], ju[pos]
            add(a + 1, l, r, c, val)
            b[a] += val[r == c].sum()
            np.add.at(Cs[l], (r, c), y0[a] * val)
            off = r != c
            np.add.at(Cs[l], (c[off], r[off]), y0[a] * val[off])
        for l, k in lps:
            cnt = min(lp_per_constraint, k)
            idx = rng.choice(k, size=cnt, replace=False)
            val = rng.standard_normal(cnt)
            add(a + 1, l, idx, idx, val)
            b[a] += val.sum()
            np.add.at(Cl[l], idx, y0[a] * val)
    for l, k in sdp:
        iu, ju = np.triu_indices(k)
        add(0, l, iu, ju, -Cs[l][iu, ju])
    for l, k in lps:
        add(0, l, np.arange(k), np.arange(k), -Cl[l])
    return Instance(m=m, blocks=[int(x) for x in blocks], c=b, k=np.concatenate(ks), l=np.concatenate(ls),
                    i=np.concatenate(is_), j=np.concatenate(js), v=np.concatenate(vs),
                    name=name or f"random block sdp {blocks} m={m} seed {seed}")


def block_arrow_sdp(nblk: int = 24, n: int = 8, m_per: int = 24, n_couple: int = 8, density: float = 0.3,
                    seed: int = 1, shuffled: bool = False) -> Instance:
    """Many SDP blocks with a sparse Schur complement: m_per constraints touch
    only block b (b = 0 .. nblk-1, in order), then n_couple constraints touch
    two random blocks each, so the Schur matrix is block-diagonal with a
    dense border (an arrowhead).  Built like `random_block_sdp` (strictly
    feasible from X = Y = I), no LP block.  shuffled: the constraints in a
    seeded random order instead (the same problem up to the numbering, whose
    Schur pattern in file order has no structure)."""
    rng = np.random.default_rng(seed)
    touch = [[b] for b in range(nblk) for _ in range(m_per)]
    for _ in range(n_couple):
        touch.append([int(x) for x in rng.choice(nblk, size=2, replace=False)])
    if shuffled:
        touch = [touch[t] for t in np.random.default_rng(seed + 1000).permutation(len(touch))]
    return random_block_sdp(len(touch), [n] * nblk, density, lp_per_constraint=0, seed=seed + 7, touch=touch,
                            name=f"block arrow sdp {nblk}x{n} m={len(touch)} seed {seed}")


def batch_block_sdp(seed: int) -> Instance:
    """One instance of the batched multi-block family: 2..4 SDP blocks of
    order U{6..40}, an LP block of U{0..12} entries (none if 0), m ~ U{10..80},
    density U(0.05, 0.2)."""
    rng = np.random.default_rng(seed)
    nsdp = int(rng.integers(2, 5))
    blocks = [int(x) for x in rng.integers(6, 41, size=nsdp)]
    nlp = int(rng.integers(0, 13))
    if nlp:
        blocks.append(-nlp)
    m = int(rng.integers(10, 81))
    dens = float(rng.uniform(0.05, 0.2))
    return random_block_sdp(m, blocks, dens, seed=seed + 1000003, name=f"batched block sdp seed {seed}")


def main(argv=None):
    """Writes a generated instance as an SDPA .dat-s file:

        python -m sdpa_b200.instances mc1  OUT.dat-s   # MaxCut G(100, 0.1), seed 1
        python -m sdpa_b200.instances lt   OUT.dat-s   # Lovasz theta G(200, 0.5), seed 1 (m = 9986)
        python -m sdpa_b200.instances rnd  OUT.dat-s   # random m = 2000, blocks {500, -50}, seed 1
        python -m sdpa_b200.instances mcb SEED OUT.dat-s  # one batched-MaxCut instance
    """
    import sys
    a = list(sys.argv[1:] if argv is None else argv)
    if len(a) == 2 and a[0] in ("mc1", "lt", "rnd"):
        it = {"mc1": lambda: maxcut(100, 0.1, 1), "lt": lambda: lovasz_theta(200, 0.5, 1),
              "rnd": lambda: random_sdp(seed=1)}[a[0]]()
        it.write(a[1])
    elif len(a) == 3 and a[0] == "mcb":
        batch_maxcut(int(a[1])).write(a[2])
    else:
        print(main.__doc__)
        return 2
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
