"""Block patterns of ChiDG Jacobians on structured hex boxes, and seeded
synthetic block values with that layout.

The pattern follows domain_matrix_t%init (src/containers/type_domain_matrix.f90:
102-632): elements in i-fastest order (src/io/mod_plot3d_utilities.f90:140-176),
per (element, time) row the interior-face blocks in face order XI_MIN, XI_MAX,
ETA_MIN, ETA_MAX, ZETA_MIN, ZETA_MAX followed by DIAG (boundary faces have no
block, :280), then for harmonic balance one hb block per other time level
(:467-491).  Subdomains ("ranks") are boxes numbered i-fastest.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib

XI_MIN, XI_MAX, ETA_MIN, ETA_MAX, ZETA_MIN, ZETA_MAX, DIAG, OTHER = range(8)

# default synthetic value model: diagonal shift, diagonal spread, face scales
# (upwind XI_MIN strongest), scale of chimera/bc/hb blocks
DEFAULT_PARAMS = (1.0, 0.6, 1.0, 0.4, 0.7, 0.4, 0.7, 0.4, 0.1)


@dataclass
class BlockPattern:
    nelem: int
    ntime: int
    elem_nvars: np.ndarray
    elem_nterms: np.ndarray
    elem_proc: np.ndarray
    blk_row_elem: np.ndarray
    blk_row_time: np.ndarray
    blk_col_elem: np.ndarray
    blk_col_time: np.ndarray
    blk_kind: np.ndarray
    blk_face: np.ndarray          # XI_MIN..ZETA_MAX, DIAG, OTHER (synthetic value model)
    shape: tuple = ()
    extra: dict = field(default_factory=dict)

    @property
    def nblocks(self) -> int:
        return int(self.blk_row_elem.size)

    def bsize(self) -> np.ndarray:
        return (self.elem_nvars * self.elem_nterms).astype(np.int64)

    def block_dims(self):
        b = self.bsize()
        return b[self.blk_row_elem], b[self.blk_col_elem]

    def value_offsets(self):
        nr, nc = self.block_dims()
        sizes = nr * nc
        off = np.zeros(self.nblocks + 1, dtype=np.int64)
        np.cumsum(sizes, out=off[1:])
        return off[:-1], int(off[-1])

    def vector_size(self) -> int:
        return int((self.bsize() * self.ntime).sum())

    def elem_offsets(self):
        sizes = self.bsize() * self.ntime
        off = np.zeros(self.nelem + 1, dtype=np.int64)
        np.cumsum(sizes, out=off[1:])
        return off

    def as_struct(self):
        """ctypes Pattern struct; keeps the arrays alive on the returned object."""
        keep = [np.ascontiguousarray(a, dtype=np.int32) for a in
                (self.elem_nvars, self.elem_nterms, self.elem_proc, self.blk_row_elem, self.blk_row_time,
                 self.blk_col_elem, self.blk_col_time, self.blk_kind)]
        p = _lib.Pattern()
        p.nelem, p.ntime, p.nblocks = self.nelem, self.ntime, self.nblocks
        ptr = lambda a: a.ctypes.data_as(_lib.I32P)
        p.elem_nvars, p.elem_nterms, p.elem_proc = ptr(keep[0]), ptr(keep[1]), ptr(keep[2])
        p.blk_row_elem, p.blk_row_time = ptr(keep[3]), ptr(keep[4])
        p.blk_col_elem, p.blk_col_time, p.blk_kind = ptr(keep[5]), ptr(keep[6]), ptr(keep[7])
        p._keep = keep
        return p


def box_pattern(nx: int, ny: int, nz: int, nvars: int, nterms: int, ntime: int = 1,
                subdomains: tuple = (1, 1, 1)) -> BlockPattern:
    """Pattern of the full Jacobian of an nx*ny*nz hex box."""
    E = nx * ny * nz
    e = np.arange(E, dtype=np.int64)
    i, j, k = e % nx, (e // nx) % ny, e // (nx * ny)
    nbr = np.full((E, 7), -1, dtype=np.int64)
    nbr[:, XI_MIN] = np.where(i > 0, e - 1, -1)
    nbr[:, XI_MAX] = np.where(i < nx - 1, e + 1, -1)
    nbr[:, ETA_MIN] = np.where(j > 0, e - nx, -1)
    nbr[:, ETA_MAX] = np.where(j < ny - 1, e + nx, -1)
    nbr[:, ZETA_MIN] = np.where(k > 0, e - nx * ny, -1)
    nbr[:, ZETA_MAX] = np.where(k < nz - 1, e + nx * ny, -1)
    nbr[:, DIAG] = e
    sx, sy, sz = subdomains
    if nx % sx or ny % sy or nz % sz:
        raise ValueError("subdomain counts must divide the box")
    proc = (i // (nx // sx)) + sx * ((j // (ny // sy)) + sy * (k // (nz // sz)))
    valid = nbr >= 0                                   # (E, 7)
    nloc = valid.sum(axis=1)                           # blocks per (e, t) row from lblks
    rows_e = np.repeat(e, ntime)                       # row order: element-major, then time
    rows_t = np.tile(np.arange(ntime), E)
    nhb = ntime - 1 if ntime > 1 else 0
    per_row = nloc[rows_e] + nhb
    R = rows_e.size
    row_start = np.zeros(R + 1, dtype=np.int64)
    np.cumsum(per_row, out=row_start[1:])
    nb = int(row_start[-1])
    bre = np.repeat(rows_e, per_row)
    brt = np.repeat(rows_t, per_row)
    bce = np.empty(nb, dtype=np.int64)
    bct = np.empty(nb, dtype=np.int64)
    bkind = np.empty(nb, dtype=np.int64)
    bface = np.empty(nb, dtype=np.int64)
    # local blocks: the valid faces of each element, element-major in face order
    elem_of, face_of = np.nonzero(valid)
    first = np.zeros(E + 1, dtype=np.int64)
    np.cumsum(nloc, out=first[1:])
    within = np.arange(elem_of.size) - first[elem_of]  # position inside the row
    for t in range(ntime):
        starts = row_start[e * ntime + t]              # (E,)
        dst = starts[elem_of] + within
        bce[dst] = nbr[elem_of, face_of]
        bct[dst] = t
        bkind[dst] = _lib.BLK_LOCAL
        bface[dst] = face_of
        if nhb:
            others = [tt for tt in range(ntime) if tt != t]
            for q, tt in enumerate(others):
                d2 = starts + nloc + q
                bce[d2] = e
                bct[d2] = tt
                bkind[d2] = _lib.BLK_HB
                bface[d2] = OTHER
    return BlockPattern(
        nelem=E, ntime=ntime,
        elem_nvars=np.full(E, nvars, dtype=np.int32), elem_nterms=np.full(E, nterms, dtype=np.int32),
        elem_proc=proc.astype(np.int32),
        blk_row_elem=bre.astype(np.int32), blk_row_time=brt.astype(np.int32),
        blk_col_elem=bce.astype(np.int32), blk_col_time=bct.astype(np.int32),
        blk_kind=bkind.astype(np.int32), blk_face=bface.astype(np.int32),
        shape=(nx, ny, nz), extra={"subdomains": tuple(subdomains)})


def with_element_orders(pat: BlockPattern, orders) -> BlockPattern:
    """The same block pattern with a polynomial order per element (ragged
    blocks: a block coupling orders p and q is nterms(p)*nvars rows by
    nterms(q)*nvars columns)."""
    orders = np.asarray(orders)
    nterms = np.array([nterms_of_order(int(o)) for o in orders], dtype=np.int32)
    return BlockPattern(nelem=pat.nelem, ntime=pat.ntime, elem_nvars=pat.elem_nvars.copy(), elem_nterms=nterms,
                        elem_proc=pat.elem_proc.copy(), blk_row_elem=pat.blk_row_elem.copy(),
                        blk_row_time=pat.blk_row_time.copy(), blk_col_elem=pat.blk_col_elem.copy(),
                        blk_col_time=pat.blk_col_time.copy(), blk_kind=pat.blk_kind.copy(), blk_face=pat.blk_face.copy(),
                        shape=pat.shape, extra=dict(pat.extra))


def nterms_of_order(p: int) -> int:
    """Legendre tensor basis size (P+1)^3 (src/chidg/type_chidg.f90:572)."""
    return (p + 1) ** 3


def synth_values(pat: BlockPattern, seed: int = 0, params=DEFAULT_PARAMS, out=None, nthreads=None) -> np.ndarray:
    """Seeded synthetic block values (packed, column-major), see csrc/synth.cpp."""
    nr, nc = pat.block_dims()
    voff, nval = pat.value_offsets()
    if out is None:
        out = np.empty(nval, dtype=np.float64)
    assert out.size >= nval and out.dtype == np.float64
    nr32 = np.ascontiguousarray(nr, dtype=np.int32)
    nc32 = np.ascontiguousarray(nc, dtype=np.int32)
    voff64 = np.ascontiguousarray(voff, dtype=np.int64)
    bt = np.ascontiguousarray(pat.blk_face, dtype=np.int32)
    prm = np.ascontiguousarray(params, dtype=np.float64)
    nthreads = nthreads or max(1, len(os.sched_getaffinity(0)))
    _lib.synth().chidg_synth_blocks(pat.nblocks, nr32.ctypes.data_as(_lib.I32P), nc32.ctypes.data_as(_lib.I32P),
                                    voff64.ctypes.data_as(_lib.I64P), bt.ctypes.data_as(_lib.I32P),
                                    C.c_uint64(seed), prm.ctypes.data_as(_lib.DP),
                                    out.ctypes.data_as(_lib.DP), int(nthreads))
    return out


def synth_vector(n: int, seed: int = 0, out=None, nthreads=None) -> np.ndarray:
    if out is None:
        out = np.empty(n, dtype=np.float64)
    nthreads = nthreads or max(1, len(os.sched_getaffinity(0)))
    _lib.synth().chidg_synth_vector(int(n), C.c_uint64(seed), out.ctypes.data_as(_lib.DP), int(nthreads))
    return out


def concat_patterns(patterns):
    """Pack independent systems block-diagonally into one pattern.

    Returns (pattern, sys_elem) where system s owns elements
    sys_elem[s]:sys_elem[s+1] of the union (the layout the batched solver
    expects).  Element ranks (elem_proc) are kept per system."""
    ntime = patterns[0].ntime
    if any(p.ntime != ntime for p in patterns):
        raise ValueError("all systems of a batch need the same number of time levels")
    eoff = np.zeros(len(patterns) + 1, dtype=np.int64)
    np.cumsum([p.nelem for p in patterns], out=eoff[1:])
    cat = lambda name, shift=False: np.concatenate(
        [getattr(p, name).astype(np.int64) + (eoff[i] if shift else 0) for i, p in enumerate(patterns)]).astype(np.int32)
    union = BlockPattern(
        nelem=int(eoff[-1]), ntime=ntime,
        elem_nvars=cat("elem_nvars"), elem_nterms=cat("elem_nterms"), elem_proc=cat("elem_proc"),
        blk_row_elem=cat("blk_row_elem", True), blk_row_time=cat("blk_row_time"),
        blk_col_elem=cat("blk_col_elem", True), blk_col_time=cat("blk_col_time"),
        blk_kind=cat("blk_kind"), blk_face=cat("blk_face"),
        shape=(), extra={"systems": len(patterns)})
    return union, eoff.astype(np.int32)
