"""ORACLE — test infrastructure only (checker, never shipped or measured).

Pure-Python restatement of the reference's :deg elimination, written with
mutable record objects like the Julia source so that it shares no code or
data layout with the product's C++ elimination:
  LLp / LLmatp            src/approxCholTypes.jl:14-39, src/approxChol.jl:102-136
  flipIndex               src/graphUtils.jl:49-55
  get_ll_col              src/approxChol.jl:354-385
  compressCol!            src/approxChol.jl:415-449
  approxChol(::LLmatp)    src/approxChol.jl:864-977
  ApproxCholPQ + ops      src/approxChol.jl:2085-2239
  sort!(…, QuickSort, o)  Julia 1.8 Base.Sort (median-of-three quicksort,
                          insertion sort for ranges of at most 21 elements)
Small graphs only (pure Python loops).  Returns the LDLinv arrays, 1-based.
"""
from __future__ import annotations

import numpy as np

from julia_rng import JuliaRng


class LLp:
    __slots__ = ("row", "val", "next", "reverse")

    def __init__(self, row, val):
        self.row = row
        self.val = val
        self.next = self
        self.reverse = self


# ---- Julia 1.8 Base.Sort.QuickSort on v[lo..hi] (1-based, inclusive) ----------

def _insertion(v, lo, hi, lt):
    for i in range(lo + 1, hi + 1):
        j = i
        x = v[i]
        while j > lo:
            if lt(x, v[j - 1]):
                v[j] = v[j - 1]
                j -= 1
                continue
            break
        v[j] = x


def _selectpivot(v, lo, hi, lt):
    mi = lo + ((hi - lo) >> 1)
    if lt(v[lo], v[mi]):
        v[mi], v[lo] = v[lo], v[mi]
    if lt(v[hi], v[lo]):
        if lt(v[hi], v[mi]):
            v[hi], v[lo], v[mi] = v[lo], v[mi], v[hi]
        else:
            v[hi], v[lo] = v[lo], v[hi]
    return v[lo]


def _partition(v, lo, hi, lt):
    pivot = _selectpivot(v, lo, hi, lt)
    i, j = lo, hi
    while True:
        i += 1
        j -= 1
        while lt(v[i], pivot):
            i += 1
        while lt(pivot, v[j]):
            j -= 1
        if i >= j:
            break
        v[i], v[j] = v[j], v[i]
    v[j], v[lo] = pivot, v[j]
    return j


def quicksort(v, lo, hi, lt):
    while lo < hi:
        if hi - lo <= 20:
            _insertion(v, lo, hi, lt)
            return
        j = _partition(v, lo, hi, lt)
        if j - lo < hi - j:
            if lo < j - 1:
                quicksort(v, lo, j - 1, lt)
            lo = j + 1
        else:
            if j + 1 < hi:
                quicksort(v, j + 1, hi, lt)
            hi = j - 1


# ---- ApproxCholPQ -------------------------------------------------------------

class PQ:
    def __init__(self, degs, n, split=1):
        self.n = n
        self.split = split
        self.prev = [0] * (n + 1)
        self.next = [0] * (n + 1)
        self.key = [0] * (n + 1)
        self.lists = [0] * (2 * split * n + 2)
        self.minlist = 1
        self.nitems = n
        for i in range(1, n + 1):
            key = degs[i]
            head = self.lists[key]
            if head > 0:
                self.prev[i], self.next[i], self.key[i] = 0, head, key
                self.prev[head] = i
            else:
                self.prev[i], self.next[i], self.key[i] = 0, 0, key
            self.lists[key] = i

    def keymap(self, x):
        k, upper = self.split * self.n, 2 * self.split * self.n + 1
        return x if x <= k else min(upper, k + x // k)

    def pop(self):
        assert self.nitems > 0, "ApproxPQ is empty"
        while self.lists[self.minlist] == 0:
            self.minlist += 1
        i = self.lists[self.minlist]
        nx = self.next[i]
        self.lists[self.minlist] = nx
        if nx > 0:
            self.prev[nx] = 0
        self.nitems -= 1
        return i

    def move(self, i, newkey, oldlist, newlist):
        pv, nx = self.prev[i], self.next[i]
        if nx > 0:
            self.prev[nx] = pv
        if pv > 0:
            self.next[pv] = nx
        else:
            self.lists[oldlist] = nx
        head = self.lists[newlist]
        if head > 0:
            self.prev[head] = i
        self.lists[newlist] = i
        self.prev[i], self.next[i], self.key[i] = 0, head, newkey

    def dec(self, i):
        oldlist = self.keymap(self.key[i])
        newlist = self.keymap(self.key[i] - 1)
        if newlist != oldlist:
            self.move(i, self.key[i] - 1, oldlist, newlist)
            if newlist < self.minlist:
                self.minlist = newlist
        else:
            self.key[i] -= 1

    def inc(self, i):
        oldlist = self.keymap(self.key[i])
        newlist = self.keymap(self.key[i] + 1)
        if newlist != oldlist:
            self.move(i, self.key[i] + 1, oldlist, newlist)
        else:
            self.key[i] += 1


def approx_chol(colptr, rowval, nzval, rng: JuliaRng):
    """colptr/rowval 1-based (Julia CSC, rows sorted), nzval weights."""
    n = len(colptr) - 1
    m = colptr[n] - 1
    # LLmatp(a)
    degs = [0] * (n + 1)
    llelems = [None] * (m + 1)
    cols = [None] * (n + 1)
    for i in range(1, n + 1):
        degs[i] = colptr[i] - colptr[i - 1]
        ind = colptr[i - 1]
        nxt = llelems[ind] = LLp(rowval[ind - 1], nzval[ind - 1])
        for ind in range(colptr[i - 1] + 1, colptr[i]):
            e = LLp(rowval[ind - 1], nzval[ind - 1])
            e.next = nxt
            llelems[ind] = e
            nxt = e
        cols[i] = nxt
    # flipIndex: position of the transposed entry
    pos = {}
    for c in range(1, n + 1):
        for ind in range(colptr[c - 1], colptr[c]):
            pos[(rowval[ind - 1], c)] = ind
    for c in range(1, n + 1):
        for ind in range(colptr[c - 1], colptr[c]):
            r = rowval[ind - 1]
            llelems[ind].reverse = llelems[pos[(c, r)]]

    pq = PQ(degs, n)
    col = [0] * (n - 1)
    ldcolptr = [0] * n
    ldrowval, ldfval = [], []
    d = [0.0] * n
    ptr_row = 1
    it = 1
    by_row = lambda x, y: x.row < y.row
    by_val = lambda x, y: x.val < y.val
    while it < n:
        i = pq.pop()
        col[it - 1] = i
        ldcolptr[it - 1] = ptr_row
        it += 1
        # get_ll_col
        colspace = [None]
        ll = cols[i]
        while ll.next is not ll:
            if ll.val > 0:
                colspace.append(ll)
            ll = ll.next
        if ll.val > 0:
            colspace.append(ll)
        ln = len(colspace) - 1
        # compressCol!
        quicksort(colspace, 1, ln, by_row)
        ptr = 0
        currow = 0
        for k in range(1, ln + 1):
            if colspace[k].row != currow:
                currow = colspace[k].row
                ptr += 1
                colspace[ptr] = colspace[k]
            else:
                colspace[ptr].val = colspace[ptr].val + colspace[k].val
                colspace[k].reverse.val = 0.0
                pq.dec(currow)
        ln = ptr
        quicksort(colspace, 1, ln, by_val)
        vals = [0.0] * (ln + 1)
        cum = [0.0] * (ln + 1)
        csum = 0.0
        for k in range(1, ln + 1):
            vals[k] = colspace[k].val
            csum = csum + colspace[k].val
            cum[k] = csum
        wdeg = csum
        col_scale = 1.0
        for jo in range(1, ln):
            ll = colspace[jo]
            w = vals[jo] * col_scale
            j = ll.row
            revj = ll.reverse
            f = w / wdeg
            vals[jo] = 0.0
            r = rng.rand() * (csum - cum[jo]) + cum[jo]
            koff = ln
            for kk in range(1, ln + 1):  # searchsortedfirst on 1..len
                if not (cum[kk] < r):
                    koff = kk
                    break
            k = colspace[koff].row
            pq.inc(k)
            new_val = f * (1.0 - f) * wdeg
            revj.row = k
            revj.val = new_val
            revj.reverse = ll
            khead = cols[k]
            cols[k] = ll
            ll.next = khead
            ll.reverse = revj
            ll.val = new_val
            ll.row = j
            col_scale = col_scale * (1.0 - f)
            omf = 1.0 - f
            wdeg = wdeg * (omf * omf)
            ldrowval.append(j)
            ldfval.append(f)
            ptr_row += 1
        ll = colspace[ln]
        w = vals[ln] * col_scale
        j = ll.row
        revj = ll.reverse
        if it < n:
            pq.dec(j)
        revj.val = 0.0
        ldrowval.append(j)
        ldfval.append(1.0)
        ptr_row += 1
        d[i - 1] = w
    ldcolptr[it - 1] = ptr_row
    return (np.array(col, np.int64), np.array(ldcolptr, np.int64), np.array(ldrowval, np.int64),
            np.array(ldfval, np.float64), np.array(d, np.float64))


# ---- fixed-order elimination: LLMatOrd + approxChol(::LLMatOrd) ---------------

class LLord:
    """Immutable column record (src/approxCholTypes.jl:42-46)."""
    __slots__ = ("row", "next", "val")

    def __init__(self, row, nxt, val):
        self.row = row
        self.next = nxt
        self.val = val


class LLcol:
    """Entry of a gathered column (src/approxCholTypes.jl:54-58)."""
    __slots__ = ("row", "ptr", "val")

    def __init__(self, row, ptr, val):
        self.row = row
        self.ptr = ptr
        self.val = val


def approx_chol_ord(colptr, rowval, nzval, rng: JuliaRng, perm=None):
    """approxChol(::LLMatOrd) (src/approxChol.jl:758-862) on LLMatOrd(a)
    (src/approxChol.jl:203-229) or LLMatOrd(a, perm) (src/approxChol.jl:265-294),
    mapped back through perm as approxchol_lapWdeg does
    (src/approxChol.jl:1712-1713).  colptr/rowval 1-based; perm 1-based or None."""
    n = len(colptr) - 1
    m = colptr[n] - 1
    if perm is None:
        invp = list(range(n + 1))
        cols_of = range(1, n)  # the reference stops at n-1
    else:
        invp = [0] * (n + 1)
        for k, v in enumerate(perm, start=1):
            invp[v] = k
        cols_of = range(1, n + 1)
    lles = [None] * (m + 1)
    cols = [0] * (n + 1)
    ptr = 1
    for i0 in cols_of:
        i = invp[i0]
        nxt = 0
        for ind in range(colptr[i0 - 1], colptr[i0]):
            j = invp[rowval[ind - 1]]
            if i < j:
                lles[ptr] = LLord(j, nxt, nzval[ind - 1])
                nxt = ptr
                ptr += 1
        cols[i] = nxt

    col = [0] * (n - 1)
    ldcolptr = [0] * n
    ldrowval, ldfval = [], []
    d = [0.0] * n
    row_ptr = 1
    for i in range(1, n):
        col[i - 1] = i
        ldcolptr[i - 1] = row_ptr
        # get_ll_col (src/approxChol.jl:387-410)
        cs = [None]
        p = cols[i]
        while p != 0:
            cs.append(LLcol(lles[p].row, p, lles[p].val))
            p = lles[p].next
        ln = len(cs) - 1
        # compressCol! (src/approxChol.jl:451-492)
        quicksort(cs, 1, ln, lambda x, y: x.row < y.row)
        k = 0
        cur = LLcol(cs[1].row, cs[1].ptr, cs[1].val)
        for q in range(2, ln + 1):
            if cs[q].row != cur.row:
                k += 1
                cs[k] = cur
                cur = LLcol(cs[q].row, cs[q].ptr, cs[q].val)
            else:
                cur = LLcol(cur.row, cur.ptr, cur.val + cs[q].val)
        k += 1
        cs[k] = cur
        ln = k
        quicksort(cs, 1, ln, lambda x, y: x.val < y.val)
        cum = [0.0] * (ln + 1)
        csum = 0.0
        for q in range(1, ln + 1):
            csum = csum + cs[q].val
            cum[q] = csum
        wdeg = csum
        col_scale = 1.0
        for jo in range(1, ln):
            c = cs[jo]
            w = c.val * col_scale
            j = c.row
            f = w / wdeg
            r = rng.rand() * (csum - cum[jo]) + cum[jo]
            koff = ln
            for kk in range(1, ln + 1):  # searchsortedfirst on 1..len
                if not (cum[kk] < r):
                    koff = kk
                    break
            kv = cs[koff].row
            new_val = w * (1.0 - f)
            if j < kv:
                lles[c.ptr] = LLord(kv, cols[j], new_val)
                cols[j] = c.ptr
            else:
                lles[c.ptr] = LLord(j, cols[kv], new_val)
                cols[kv] = c.ptr
            col_scale = col_scale * (1.0 - f)
            wdeg = wdeg - 2 * w + w * w / wdeg
            ldrowval.append(j)
            ldfval.append(f)
            row_ptr += 1
        c = cs[ln]
        ldrowval.append(c.row)
        ldfval.append(1.0)
        row_ptr += 1
        d[i - 1] = c.val * col_scale
    ldcolptr[n - 1] = row_ptr
    col = np.array(col, np.int64)
    rowv = np.array(ldrowval, np.int64)
    d = np.array(d, np.float64)
    if perm is not None:
        p = np.asarray(perm, np.int64)
        col = p[col - 1]
        rowv = p[rowv - 1]
        d = d[np.asarray(invp[1:], np.int64) - 1]
    return col, np.array(ldcolptr, np.int64), rowv, np.array(ldfval, np.float64), d


# ---- split/merge elimination: LLmatp(a, split) + approxChol(a, split, merge) ---

def approx_chol_split(colptr, rowval, nzval, rng: JuliaRng, split=2, merge=2):
    """approxChol(::LLmatp, split, merge) (src/approxChol.jl:979-1157) on
    LLmatp(a, split) (src/approxChol.jl:138-183) with compressAvgCol!
    (src/approxChol.jl:541-600).  colptr/rowval 1-based.  merge < 1 is
    approxChol(::LLmatp, split) (src/approxChol.jl:1162-1322), whose avgCol!
    (src/approxChol.jl:497-533) is compressAvgCol! with no cap reached."""
    if merge < 1:
        merge = float("inf")
    n = len(colptr) - 1
    m = colptr[n] - 1
    # LLmatp(a, split): llelems[split*(ind-1)+k], k = 1..split
    degs = [0] * (n + 1)
    llelems = [None] * (split * m + 1)
    cols = [None] * (n + 1)
    for i in range(1, n + 1):
        degs[i] = split * (colptr[i] - colptr[i - 1])
        ind = colptr[i - 1]
        j = rowval[ind - 1]
        v = nzval[ind - 1] / split
        llpend = LLp(j, v)
        llelems[split * ind] = llpend
        nxt = llpend
        for k in range(1, split):
            e = LLp(j, v)
            e.next = nxt
            llelems[split * (ind - 1) + k] = e
            nxt = e
        for ind in range(colptr[i - 1] + 1, colptr[i]):
            j = rowval[ind - 1]
            v = nzval[ind - 1] / split
            for k in range(1, split + 1):
                e = LLp(j, v)
                e.next = nxt
                llelems[split * (ind - 1) + k] = e
                nxt = e
        cols[i] = nxt
    pos = {}
    for c in range(1, n + 1):
        for ind in range(colptr[c - 1], colptr[c]):
            pos[(rowval[ind - 1], c)] = ind
    for c in range(1, n + 1):
        for ind in range(colptr[c - 1], colptr[c]):
            flip = pos[(c, rowval[ind - 1])]
            for k in range(1, split + 1):
                llelems[split * (ind - 1) + k].reverse = llelems[split * (flip - 1) + k]

    pq = PQ(degs, n, split)
    col = [0] * (n - 1)
    ldcolptr = [0] * n
    ldrowval, ldfval = [], []
    d = [0.0] * n
    row_ptr = 1
    it = 1
    while it < n:
        i = pq.pop()
        col[it - 1] = i
        ldcolptr[it - 1] = row_ptr
        it += 1
        cs = [None]
        ll = cols[i]
        while ll.next is not ll:
            if ll.val > 0:
                cs.append(ll)
            ll = ll.next
        if ll.val > 0:
            cs.append(ll)
        ln = len(cs) - 1
        # compressAvgCol!
        quicksort(cs, 1, ln, lambda x, y: x.row < y.row)
        cur, nxt, ptr = 1, 1, 0
        while nxt <= ln and cs[cur].row == cs[nxt].row:
            nxt += 1
        while cur <= ln:
            num = nxt - cur
            mul_sum = 0.0
            for q in range(cur, nxt):
                mul_sum += cs[q].val
            if num <= merge:
                nv = mul_sum / num
                for q in range(cur, nxt):
                    cs[q].val = nv
                    cs[q].reverse.val = nv
                    ptr += 1
                    cs[ptr] = cs[q]
            else:
                nv = mul_sum / merge
                for q in range(cur, cur + merge):
                    cs[q].val = nv
                    cs[q].reverse.val = nv
                    ptr += 1
                    cs[ptr] = cs[q]
                currow = cs[cur].row
                for q in range(cur + merge, nxt):
                    cs[q].reverse.val = 0.0
                    pq.dec(currow)
            cur = nxt
            while nxt <= ln and cs[cur].row == cs[nxt].row:
                nxt += 1
        ln = ptr
        quicksort(cs, 1, ln, lambda x, y: (x.val, x.row) < (y.val, y.row))
        vals = [0.0] * (ln + 1)
        csum = 0.0
        for q in range(1, ln + 1):
            csum = csum + cs[q].val
            vals[q] = cs[q].val
        csr = [0.0] * (ln + 2)
        crev = 0.0
        for q in range(ln, 0, -1):
            crev += cs[q].val
            csr[q] = crev
        wdeg = csum
        col_scale = 1.0
        next_edge = 1
        final_d = 0.0
        for jo in range(1, ln):
            is_new = jo == next_edge
            while next_edge <= ln and cs[jo].row == cs[next_edge].row:
                next_edge += 1
            if next_edge == ln + 1:
                q = jo
                while q <= ln - 1:
                    e = cs[q]
                    final_d += vals[q] * col_scale
                    if it < n:
                        pq.dec(e.row)
                    e.reverse.val = 0.0
                    q += 1
                break
            ll = cs[jo]
            w = vals[jo] * col_scale
            j = ll.row
            revj = ll.reverse
            f = w / wdeg
            vals[jo] = 0.0
            r = rng.rand() * csr[next_edge]
            koff = 0  # searchsortedlast under the reverse order: last q with csr[q] >= r
            for q in range(1, ln + 1):
                if not (csr[q] < r):
                    koff = q
            k = cs[koff].row
            pq.inc(k)
            new_val = ll.val * csr[next_edge] / csum
            revj.row = k
            revj.val = new_val
            revj.reverse = ll
            khead = cols[k]
            cols[k] = ll
            ll.next = khead
            ll.reverse = revj
            ll.val = new_val
            ll.row = j
            if is_new:
                ldrowval.append(j)
                ldfval.append(f)
                row_ptr += 1
            else:
                ldfval[-1] = ldfval[-1] + f
            if jo == next_edge - 1:
                f = ldfval[-1]
                col_scale = col_scale * (1.0 - f)
                wdeg = wdeg * ((1.0 - f) * (1.0 - f))
        ll = cs[ln]
        final_d += vals[ln] * col_scale
        j = ll.row
        if it < n:
            pq.dec(j)
        ll.reverse.val = 0.0
        ldrowval.append(j)
        ldfval.append(1.0)
        row_ptr += 1
        d[i - 1] = final_d
    ldcolptr[it - 1] = row_ptr
    return (np.array(col, np.int64), np.array(ldcolptr, np.int64), np.array(ldrowval, np.int64),
            np.array(ldfval, np.float64), np.array(d, np.float64))
