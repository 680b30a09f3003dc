"""CPU restatement of the reference's graph input (TEST INFRASTRUCTURE ONLY).

Only tests/ may import this module; the product path never does.  Parity is
unpinned: the reference ships no graph files or loader tests, so the cases in
tests/test_graph_io_oracle.py are hand-computed from the rules below.

* ``parse_mtx`` follows load_mtx_graph (app/io/io_mtx.cpp:204-333) with the
  banner fields of get_mm_metadata (:22-56): a character scanner over the
  whole file, digits-only integers (io_common fast_atoi), 1-based ids,
  ``%`` comment lines anywhere, an error on a line holding one value.
* ``construct_from_edgelist`` follows io_mtx.cpp:95-201: self loops and (when
  weighted) zero weights dropped; non-symmetric lists keep the first copy of
  each unordered pair (is_new_entry, :60-93); both directions stored; rows
  sorted by column.  Equal (row, column) entries of a symmetric list keep
  input order (a stable sort), where the reference leaves them in an
  unspecified order.
* ``parse_metis`` follows load_metis_graph (app/io/io_metis.cpp:64-181).
* ``load_graph`` dispatches on the ``.mtx`` suffix (io_mtx.cpp:336-345).

Each function raises ``ValueError`` where the reference prints FATAL ERROR.
"""
from __future__ import annotations

import numpy as np

OBJ_MOD, OBJ_WMOD, OBJ_CPM, OBJ_NLCC, OBJ_LCC = 0, 1, 2, 3, 4


class _Scanner:
    def __init__(self, data: bytes):
        self.s = data if data.endswith(b"\n") else data + b"\n"
        self.i = 0
        self.n = len(self.s)

    def next_line(self):
        j = self.s.find(b"\n", self.i)
        self.i = self.n if j < 0 else j + 1

    def atoi(self) -> int:
        j = self.i
        while j < self.n and 48 <= self.s[j] <= 57:
            j += 1
        v = int(self.s[self.i:j]) if j > self.i else 0
        self.i = j
        return v

    def isdigit(self) -> bool:
        return 48 <= self.s[self.i] <= 57

    def header(self, count: int):
        while self.i < self.n and self.s[self.i] == ord("%"):
            self.next_line()
        while self.i < self.n and not self.isdigit():
            self.i += 1
        out = [0] * count
        k = 0
        while k < count:
            out[k] = self.atoi()
            while self.i < self.n and not self.isdigit():
                if self.s[self.i] == ord("\n"):
                    k = count
                    self.i += 1
                    break
                self.i += 1
            k += 1
        return out


def _mm_fields(data: bytes):
    line = data.split(b"\n", 1)[0].decode("latin-1")
    fields, cur = [], ""
    for c in line + " ":
        if c.isalnum() and c.isascii():
            cur += c
        else:
            if cur and len(fields) < 5:
                fields.append(cur)
            cur = ""
    fields += [""] * (5 - len(fields))
    return fields


def parse_mtx(data: bytes, uniform: bool):
    """-> (n, src, dst, w or None, symmetric, uniform)"""
    f = _mm_fields(data)
    if f[2] != "coordinate":
        raise ValueError("non-coordinate Matrix Market file")
    pattern, integer, symmetric = f[3] == "pattern", f[3] == "integer", f[4] == "symmetric"
    if not pattern and not integer:
        uniform = True
    if not symmetric:
        uniform = True
    sc = _Scanner(data)
    n, n2, m, _ = sc.header(4)
    if n != n2:
        raise ValueError("bipartite Matrix Market file")
    weighted = not uniform and not pattern
    src = np.zeros(m, np.int64)
    dst = np.zeros(m, np.int64)
    w = np.zeros(m, np.int64) if weighted else None
    read, state = 0, 0
    s = sc.s
    while sc.i < sc.n:
        while sc.i < sc.n and not sc.isdigit():
            if s[sc.i] == ord("%"):
                sc.next_line()
                continue
            if s[sc.i] == ord("\n") and state != 0:
                raise ValueError("line with exactly one value")
            sc.i += 1
        if sc.i >= sc.n:
            break
        if read >= m:
            raise ValueError("more entries than the header states")
        v = sc.atoi()
        if state == 0:
            src[read] = v - 1
            state = 1
        elif state == 1:
            dst[read] = v - 1
            if not weighted:
                state = 0
                read += 1
                sc.next_line()
            else:
                state = 2
        else:
            w[read] = v
            read += 1
            state = 0
            sc.next_line()
    if read != m:
        raise ValueError("entry count differs from the header")
    if m and (src.min() < 0 or dst.min() < 0 or src.max() >= n or dst.max() >= n):
        raise ValueError("entry index out of range")
    return n, src, dst, w, symmetric, not weighted


def construct_from_edgelist(n: int, src, dst, w, symmetric: bool):
    """-> (rowptr int64, col int32, w int32 or None)"""
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    keep = src != dst
    if w is not None:
        keep &= np.asarray(w) != 0
    if not symmetric:
        lo, hi = np.minimum(src, dst), np.maximum(src, dst)
        pair = lo * max(n, 1) + hi
        first = np.zeros(len(src), bool)
        kept = np.flatnonzero(keep)
        _, idx = np.unique(pair[kept], return_index=True)
        first[kept[idx]] = True
        keep &= first
    s, d = src[keep], dst[keep]
    # entry j contributes (s, d) then (d, s): the interleaved order a stable sort keeps
    rows = np.stack([s, d], 1).reshape(-1)
    cols = np.stack([d, s], 1).reshape(-1)
    order = np.lexsort((cols, rows))  # stable
    rows, cols = rows[order], cols[order]
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    wout = None
    if w is not None:
        wk = np.asarray(w, np.int64)[keep]
        wout = np.stack([wk, wk], 1).reshape(-1)[order].astype(np.int32)
    return rowptr, cols.astype(np.int32), wout


def parse_metis(data: bytes, uniform: bool):
    """-> (rowptr int64, col int32, w int32 or None, uniform)"""
    sc = _Scanner(data)
    n, m, fmt, ncon = sc.header(4)
    if fmt not in (0, 1):
        raise ValueError("unsupported METIS format flags")
    if ncon != 0:
        raise ValueError("unsupported METIS ncon")
    has_ew = fmt == 1
    if not has_ew:
        uniform = True
    weighted = has_ew and not uniform
    rowptr = np.zeros(n + 1, np.int64)
    col = np.zeros(2 * m, np.int64)
    w = np.zeros(2 * m, np.int64) if weighted else None
    edges = rows = 0
    is_value = False
    s = sc.s
    while sc.i < sc.n:
        while sc.i < sc.n and not sc.isdigit():
            if s[sc.i] == ord("%"):
                sc.next_line()
                continue
            if s[sc.i] == ord("\n") and rows < n:
                rows += 1
                rowptr[rows] = edges
            sc.i += 1
        if sc.i >= sc.n:
            break
        v = sc.atoi()
        if not is_value:
            if edges >= 2 * m:
                raise ValueError("more adjacency entries than the header states")
            col[edges] = v - 1
            if not has_ew:
                edges += 1
        else:
            if weighted:
                w[edges] = v
            edges += 1
        if has_ew:
            is_value = not is_value
    if rows != n or edges != 2 * m:
        raise ValueError("line or adjacency count differs from the header")
    if edges and (col.min() < 0 or col.max() >= n):
        raise ValueError("neighbour id out of range")
    return rowptr, col.astype(np.int32), None if w is None else w.astype(np.int32), not weighted


def load_graph(path: str, objective: int):
    """-> (rowptr, col, w or None, edge_uniform); Mod and CPM ignore weights
    (app/objective_helpers.hpp:24-29)."""
    uniform = objective in (OBJ_MOD, OBJ_CPM)
    with open(path, "rb") as fh:
        data = fh.read()
    if str(path).endswith(".mtx"):
        n, src, dst, w, sym, uni = parse_mtx(data, uniform)
        rowptr, col, wout = construct_from_edgelist(n, src, dst, w, sym)
        return rowptr, col, wout, uni
    rowptr, col, w, uni = parse_metis(data, uniform)
    return rowptr, col, w, uni
