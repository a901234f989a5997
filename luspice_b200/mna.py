"""Seeded synthetic SPICE MNA matrices (no netlists ship with the reference).

Every generator stamps circuit elements into a modified-nodal-analysis
matrix and keeps the element list, so Newton-step value perturbations are
re-stamped element by element (the pattern never changes between them).

Workloads (base seed 42, seed = 42 + matrix index):
  analog(989)        900 nodes + 89 voltage-source branch rows (zero
                     diagonal, +-1 incidence, - terminal ground or a nearby
                     node); ~4 resistor stamps per node
                     (to nodes of the same subcircuit: node numbers within
                     a window of 4),
                     G log-uniform [1e-6, 1e-1] S; capacitor companions C/h,
                     C log-uniform [1e-15, 1e-11] F, h = 1e-9 s; 150
                     unsymmetric MOSFET gm/gds stamps, gm log-uniform
                     [1e-5, 1e-2], on random node pairs (log-uniform
                     distance 1..32; ~30 terminals per circuit uniformly
                     random across it); gmin 1e-12 on node diagonals;
                     x_true ~ U[-1, 1], b = A x_true.
  power_grid()       63 x 64 resistive mesh (segment G log-uniform [0.1, 10])
                     + 18 Vdd pad branch rows; decap C log-uniform
                     [1e-12, 1e-10] F, h = 1e-10 s; load currents in b
                     uniform [0, 1e-3] A.  n = 4050.
  large_circuit()    n = 40,000, ~200k entries: the analog netlist plus
                     supply nets coupling to 2% of the nodes (~800 entries in
                     each such row and column); conductance and capacitor
                     values log-uniform over [1e-12, 1e3] (MOSFET gm stays
                     in [1e-5, 1e-2]: transconductances spanning 15 decades
                     make partial pivoting leave the fill-reducing order).
Perturbation: every element value times exp(sigma * N(0, 1)), sigma = 0.1.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

FP16_MIN_NORMAL = 2.0 ** -14


@dataclass
class MNAMatrix:
    name: str
    n: int
    Ap: np.ndarray           # int32 [n+1], CSC, rows ascending per column
    Ai: np.ndarray           # int32 [nnz]
    Ax: np.ndarray           # float64 [nnz], nominal values
    stamp: sp.csr_matrix     # [nnz x n_elem]: entry = stamp @ elem_val + const
    const: np.ndarray        # [nnz] element-independent entries (incidence)
    elem_val: np.ndarray     # [n_elem] nominal element values
    b: np.ndarray            # [n]
    x_true: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.Ap[-1])

    def values(self, factors: np.ndarray | None = None) -> np.ndarray:
        ev = self.elem_val if factors is None else self.elem_val * factors
        return np.asarray(self.stamp @ ev).ravel() + self.const

    def perturbed(self, count: int, seed: int, sigma: float = 0.1) -> np.ndarray:
        """count value sets (count x nnz), element values x exp(sigma N(0,1))."""
        rng = np.random.default_rng(seed)
        out = np.empty((count, self.nnz))
        for t in range(count):
            out[t] = self.values(np.exp(sigma * rng.standard_normal(self.elem_val.size)))
        return out

    def csr(self, values: np.ndarray | None = None) -> sp.csr_matrix:
        v = self.Ax if values is None else values
        return sp.csc_matrix((v, self.Ai, self.Ap), shape=(self.n, self.n)).tocsr()

    def matvec(self, x: np.ndarray, values: np.ndarray | None = None) -> np.ndarray:
        v = self.Ax if values is None else values
        return sp.csc_matrix((v, self.Ai, self.Ap), shape=(self.n, self.n)) @ x


class _Stamper:
    """Collects (row, col, element, coefficient) stamps; element -1 = constant."""

    def __init__(self, n: int):
        self.n = n
        self.r: list[np.ndarray] = []
        self.c: list[np.ndarray] = []
        self.e: list[np.ndarray] = []
        self.k: list[np.ndarray] = []
        self.vals: list[np.ndarray] = []
        self.nelem = 0

    def elements(self, values: np.ndarray) -> np.ndarray:
        ids = np.arange(self.nelem, self.nelem + values.size)
        self.nelem += values.size
        self.vals.append(np.asarray(values, dtype=np.float64))
        return ids

    def add(self, rows, cols, elems, coefs):
        rows = np.asarray(rows)
        cols = np.asarray(cols)
        keep = (rows >= 0) & (cols >= 0)
        self.r.append(rows[keep].astype(np.int64))
        self.c.append(cols[keep].astype(np.int64))
        self.e.append(np.broadcast_to(np.asarray(elems), rows.shape)[keep].astype(np.int64))
        self.k.append(np.broadcast_to(np.asarray(coefs, dtype=np.float64), rows.shape)[keep])

    def conductance(self, a, b, elems):
        """Two-terminal conductance between nodes a and b (-1 = ground)."""
        self.add(a, a, elems, 1.0)
        self.add(b, b, elems, 1.0)
        self.add(a, b, elems, -1.0)
        self.add(b, a, elems, -1.0)

    def vccs(self, d, s, g, elems):
        """Transconductance gm: current into d out of s controlled by v(g)-v(s)."""
        self.add(d, g, elems, 1.0)
        self.add(d, s, elems, -1.0)
        self.add(s, g, elems, -1.0)
        self.add(s, s, elems, 1.0)

    def branch(self, row, p, m):
        """Voltage-source branch row: +-1 incidence, no diagonal."""
        one = -np.ones_like(np.asarray(row))
        self.add(p, row, one, 1.0)
        self.add(row, p, one, 1.0)
        self.add(m, row, one, -1.0)
        self.add(row, m, one, -1.0)

    def build(self, name: str, rng: np.random.Generator, rhs=None, meta=None) -> MNAMatrix:
        n = self.n
        r = np.concatenate(self.r)
        c = np.concatenate(self.c)
        e = np.concatenate(self.e)
        k = np.concatenate(self.k)
        elem_val = np.concatenate(self.vals) if self.vals else np.zeros(0)
        key = c * n + r
        uniq, inv = np.unique(key, return_inverse=True)
        nnz = uniq.size
        Ai = (uniq % n).astype(np.int32)
        cols = (uniq // n).astype(np.int64)
        Ap = np.zeros(n + 1, dtype=np.int64)
        np.add.at(Ap, cols + 1, 1)
        Ap = np.cumsum(Ap).astype(np.int32)
        isel = e >= 0
        stamp = sp.csr_matrix((k[isel], (inv[isel], e[isel])), shape=(nnz, max(self.nelem, 1)))
        const = np.zeros(nnz)
        np.add.at(const, inv[~isel], k[~isel])
        if self.nelem == 0:
            elem_val = np.zeros(1)
        m = MNAMatrix(name=name, n=n, Ap=Ap, Ai=Ai, Ax=np.zeros(nnz), stamp=stamp, const=const,
                      elem_val=elem_val, b=np.zeros(n), meta=dict(meta or {}))
        m.Ax = m.values()
        if rhs is None:
            x_true = rng.uniform(-1.0, 1.0, n)
            m.x_true = x_true
            m.b = m.matvec(x_true)
        else:
            m.b = np.asarray(rhs, dtype=np.float64)
        return m


def _logu(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def _distinct_pairs(rng, nodes, count):
    a = rng.integers(0, nodes, count)
    b = rng.integers(0, nodes - 1, count)
    b = np.where(b >= a, b + 1, b)
    return a, b


def analog(n_total: int = 989, seed: int = 42, value_range: tuple[float, float] | None = None,
           name: str | None = None, local: int = 4, physical_gm: bool = False) -> MNAMatrix:
    """Analog-circuit MNA matrix (see module doc); value_range replaces the
    element-value distributions by log-uniform over that range (MOSFET gm
    too, unless physical_gm keeps it in [1e-5, 1e-2])."""
    rng = np.random.default_rng(seed)
    n_br = max(1, int(round(n_total * 89 / 989)))
    nn = n_total - n_br
    n_mos = max(1, int(round(150 * nn / 900)))
    st = _Stamper(n_total)

    def vals(lo, hi, size):
        if value_range is not None:
            return _logu(rng, value_range[0], value_range[1], size)
        return _logu(rng, lo, hi, size)

    # ~4 resistor stamps per node: two resistors from each node to nodes of
    # the same subcircuit (a window of `local` node numbers), as netlists
    # number the nodes of a cell together.
    a = np.repeat(np.arange(nn), 2)
    bnode = (a + rng.integers(1, local + 1, a.size)) % nn
    st.conductance(a, bnode, st.elements(vals(1e-6, 1e-1, a.size)))
    # Capacitor companions: every node to ground, a quarter between nodes of
    # the same subcircuit.
    h = 1e-9
    nodes = np.arange(nn)
    st.conductance(nodes, -np.ones(nn, dtype=np.int64),
                   st.elements(vals(1e-15, 1e-11, nn) / h if value_range is None else vals(0, 0, nn)))
    ca = rng.integers(0, nn, nn // 4)
    cb = (ca + rng.integers(1, local + 1, ca.size)) % nn
    st.conductance(ca, cb, st.elements(vals(1e-15, 1e-11, ca.size) / h if value_range is None
                                       else vals(0, 0, ca.size)))
    # MOSFETs: gm (unsymmetric) and gds between drain and source.  Gate and
    # source are random nodes at a log-uniform distance (1..32) from the
    # drain; about 30 terminals per circuit (one in ten at n = 989) are
    # uniformly random nodes anywhere in the circuit.
    p_global = min(0.1, 30.0 / (2.0 * n_mos))

    def partner(base):
        dist = np.floor(np.exp(rng.uniform(0.0, np.log(min(32.0, max(2.0, nn / 2.0))), base.size)))
        sign = np.where(rng.random(base.size) < 0.5, -1, 1)
        near = (base + sign * np.maximum(dist.astype(np.int64), 1)) % nn
        return np.where(rng.random(base.size) < p_global, rng.integers(0, nn, base.size), near)

    d = rng.integers(0, nn, n_mos)
    g = partner(d)
    s = partner(d)
    s = np.where(s == g, (s + 1) % nn, s)
    s = np.where(s == d, (d + 2) % nn, s)
    g = np.where(g == d, (d + 1) % nn, g)
    gm = _logu(rng, 1e-5, 1e-2, n_mos) if physical_gm else vals(1e-5, 1e-2, n_mos)
    st.vccs(d, s, g, st.elements(gm))
    st.conductance(d, s, st.elements(gm / rng.uniform(10.0, 100.0, n_mos)))
    # gmin on every node diagonal.
    st.add(nodes, nodes, st.elements(np.full(nn, 1e-12)), 1.0)
    # Voltage sources: unique + terminals; - terminal ground or a nearby node
    # that is no source's + terminal (so sources never form a loop).
    perm = rng.permutation(nn)
    plus = perm[:n_br]
    is_plus = np.zeros(nn, bool)
    is_plus[plus] = True
    free = np.flatnonzero(~is_plus)
    near = (plus + rng.integers(1, local + 1, n_br)) % nn
    pos = np.searchsorted(free, near) % max(1, free.size)
    minus = np.where(rng.random(n_br) < 0.5, -1, free[pos])
    rows = nn + np.arange(n_br)
    st.branch(rows, plus, minus)
    return st.build(name or f"analog{n_total}", rng,
                    meta={"nodes": nn, "branches": n_br, "mosfets": n_mos, "seed": seed})


def power_grid(rows: int = 63, cols: int = 64, pads: int = 18, seed: int = 42) -> MNAMatrix:
    """Power-grid MNA matrix (see module doc)."""
    rng = np.random.default_rng(seed)
    nn = rows * cols
    n = nn + pads
    st = _Stamper(n)
    idx = np.arange(nn).reshape(rows, cols)
    ha, hb = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    va, vb = idx[:-1, :].ravel(), idx[1:, :].ravel()
    a = np.concatenate([ha, va])
    b = np.concatenate([hb, vb])
    st.conductance(a, b, st.elements(_logu(rng, 0.1, 10.0, a.size)))
    h = 1e-10
    st.conductance(np.arange(nn), -np.ones(nn, dtype=np.int64),
                   st.elements(_logu(rng, 1e-12, 1e-10, nn) / h))
    # Pads on a 3 x 6 lattice of the mesh.
    pr = np.linspace(0, rows - 1, 3).round().astype(int)
    pc = np.linspace(0, cols - 1, pads // 3).round().astype(int)
    pad_nodes = np.array([idx[r, c] for r in pr for c in pc])[:pads]
    st.branch(nn + np.arange(pads), pad_nodes, -np.ones(pads, dtype=np.int64))
    rhs = np.zeros(n)
    rhs[:nn] = -rng.uniform(0.0, 1e-3, nn)
    rhs[nn:] = 1.0
    return st.build(f"power_grid{n}", rng, rhs=rhs, meta={"mesh": (rows, cols), "pads": pads, "seed": seed})


def large_circuit(n_total: int = 40000, seed: int = 42, supply_nets: int = 4,
                  coupling: float = 0.02) -> MNAMatrix:
    """Large unsymmetric circuit with supply nets (see module doc)."""
    rng = np.random.default_rng(seed)
    base = analog(n_total - supply_nets, seed=seed, value_range=(1e-12, 1e3),
                  name=f"large{n_total}", physical_gm=True)
    # Rebuild with extra supply-net rows/columns appended.
    n = n_total
    st = _Stamper(n)
    # Re-stamp the base entries as fixed-coefficient elements (one element per
    # entry) so perturbations still act entry-wise on them.
    cols = np.repeat(np.arange(base.n), np.diff(base.Ap))
    st.add(base.Ai, cols, st.elements(base.Ax), 1.0)
    nodes = base.meta["nodes"]
    k = int(round(coupling * nodes))
    for s in range(supply_nets):
        net = base.n + s
        taps = rng.choice(nodes, k, replace=False)
        st.conductance(taps, np.full(k, net), st.elements(_logu(rng, 1e-12, 1e3, k)))
        st.add([net], [net], st.elements(_logu(rng, 1e-12, 1e3, 1)), 1.0)
    m = st.build(f"large{n_total}", rng, meta={"supply_nets": supply_nets, "taps": k, "seed": seed})
    a = np.abs(m.Ax[m.Ax != 0])
    m.meta["frac_below_fp16_normal"] = float(np.mean(a < FP16_MIN_NORMAL)) if a.size else 0.0
    return m


def ill_conditioned(m: MNAMatrix, seed: int, width: int = 8, scale: float = 1e-14) -> np.ndarray:
    """Values of an ill-conditioned Newton step on m's pattern: every element
    touching one subcircuit (a window of `width` node rows) is scaled by
    `scale`, and one further node keeps only its gmin (all its other
    elements are scaled by 1e-30)."""
    rng = np.random.default_rng(seed)
    nodes = int(m.meta.get("nodes", m.n))
    i0 = int(rng.integers(0, max(1, nodes - width - 1)))
    rows = np.repeat(np.arange(m.nnz), np.diff(m.stamp.indptr))
    elems = m.stamp.indices
    entry_row = m.Ai[rows]
    fac = np.ones(m.elem_val.size)
    touch = np.unique(elems[(entry_row >= i0) & (entry_row < i0 + width)])
    fac[touch] = scale
    lone = i0 + width
    gmin = m.elem_val == 1e-12
    touch2 = np.unique(elems[entry_row == lone])
    fac[touch2[~gmin[touch2]]] = 1e-30
    return m.values(fac)


SERVING_KINDS = ("analog", "grid", "supply")


def serving_class(kind: str, n: int, seed: int) -> MNAMatrix:
    """One pattern class of the serving workload, about n unknowns: "analog"
    (the n = 989 generator at size n), "grid" (a power-grid mesh of about n
    nodes with about n / 225 pads) or "supply" (the analog netlist with supply nets,
    the n = 40,000 generator at size n)."""
    if kind == "analog":
        return analog(int(n), seed)
    if kind == "grid":
        pads = 3 * max(1, int(n) // 675)      # a 3 x (pads / 3) lattice of pads
        rows = max(2, int(np.sqrt(max(4, int(n) - pads))))
        cols = max(2, (int(n) - pads) // rows)
        return power_grid(rows, cols, pads, seed)
    if kind == "supply":
        return large_circuit(max(int(n), 200), seed)
    raise ValueError(kind)


def serving_classes(count: int = 64, lo: int = 113, hi: int = 40000, seed: int = 42) -> list[tuple[str, int]]:
    """(kind, n) of the serving workload's pattern classes: n log-uniform in
    [lo, hi], the three generators in turn."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    return [(SERVING_KINDS[i % 3], int(n)) for i, n in enumerate(ns)]


def batch_sizes(count: int = 512, lo: int = 100, hi: int = 5000, seed: int = 42) -> np.ndarray:
    """Matrix sizes of the uneven batch: n ~ U[lo, hi] from the base seed."""
    return np.random.default_rng(seed).integers(lo, hi + 1, count)
