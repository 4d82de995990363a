"""The reference's own aggregation -- make_aggregation with its priority queue
(Make_amg_matrix.f90:113-222; remove_enter_quedeep / remove_que / enter_que, :633-768) --
restated in the oracle (heap_aggregate in oracle/msg123_oracle.c) as a structural known
answer beside the MIS-2 aggregation the CUDA library runs.

* a chain of 8 cells worked by hand through the queue;
* a second, independent restatement below (a Python dict-based queue that reproduces the
  array heap's moves) on the strength graphs of two heterogeneous blocks, node for node;
* the two hierarchies side by side on the same Jacobians: aggregates, nodes left out of
  every aggregate, coarse nnz per row, and BiCGStab iterations with each V-cycle.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle


def _strength(d, lu, offind, offrow, theta):
    """make_grapfilt's strong entries (Make_amg_matrix.f90:86-104): the CSR positions k of
    row i with lu_k^2 > |d_i d_j theta^2| and d_i d_j lu_k > 0, in CSR order."""
    th2 = float(np.float32(theta)) ** 2
    n = len(d)
    out = []
    for i in range(n):
        row = []
        for k in range(offind[i], offind[i + 1]):
            j = offrow[k]
            dd = d[i] * d[j]
            if lu[k] * lu[k] > abs(dd * th2) and dd * lu[k] > 0.0:
                row.append(j)
        out.append(row)
    return out


def heap_aggregation(strong):
    """The queue of make_aggregation, positions 1..size: remove_que moves the larger child
    (the right one only when strictly larger) into the hole until the hole has no queued
    child; enter_que swaps a node above its parent while the parent's priority is strictly
    smaller.  Returns 0-based aggregates, -1 for nodes outside every aggregate."""
    n = len(strong)
    flag, node, pos = {}, {}, [0] * n
    size = 0
    for i in range(n):
        if strong[i]:
            size += 1
            flag[size], node[size], pos[i] = 1, i, size

    def remove(v):
        q = pos[v]
        flag[q], node[q] = 0, None
        c = 2 * q
        while c <= size:
            if c + 1 <= size and flag.get(c + 1, 0) > flag.get(c, 0):
                c += 1
            if flag.get(c, 0) == 0:
                break
            flag[q], node[q] = flag[c], node[c]
            pos[node[q]] = q
            flag[c], node[c] = 0, None
            q, c = c, 2 * c
        pos[v] = 0

    def raise_(v):
        q = pos[v]
        while q > 1 and flag[q // 2] < flag[q]:
            p = q // 2
            flag[p], flag[q] = flag[q], flag[p]
            node[p], node[q] = node[q], node[p]
            pos[node[p]], pos[node[q]] = p, q
            q = p

    num = [0] * n
    mark = [None] * n
    nc = 0
    while size and flag.get(1, 0):
        root = node[1]
        nc += 1
        num[root] = nc
        for j in strong[root]:
            num[j] = nc
            if pos[j]:
                remove(j)
            mark[j] = root
        remove(root)
        mark[root] = root
        ring2 = []
        for j in strong[root]:
            for l2 in strong[j]:
                if mark[l2] != root:
                    mark[l2] = root
                    ring2.append(l2)
                    if pos[l2]:
                        remove(l2)
        for j in ring2:
            for l3 in strong[j]:
                if mark[l3] != root:
                    mark[l3] = root
                    if pos[l3]:
                        flag[pos[l3]] += 1
                        raise_(l3)
    for i in range(n):          # aggre_check: the first adoption ends the scan
        hit = next((j for j in strong[i] if num[j] > 0), None)
        if hit is not None:
            num[i] = num[hit]
            break
    return [v - 1 for v in num]


def _system(shape, seed, **kw):
    p = make_config("hetero", shape=shape, seed=seed, precon_type=1, ref_quirks=0, **kw)
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.003 * np.random.default_rng(seed).standard_normal(p.ncalc), delt=1800.0)
    d, lu, r = o.make_matvec()
    return p, o, d, lu, r


def test_chain_by_hand():
    """8 cells in a row, d = -2, every off-diagonal +1 (all strong).  Root 0 takes {0,1};
    cell 2 (distance 2) leaves the queue; cell 3 (distance 3) rises to priority 2 and is
    the next root, taking {2,3,4}; cell 5 leaves, cell 6 rises and takes {5,6,7}."""
    p = make_config("hetero", shape=(8, 1, 1), seed=4, precon_type=1, ref_quirks=0, amg_coarse_max=2)
    o = Oracle(p)
    o.init_state()
    o.set_aggregation(1)
    d, lu = np.full(o.n, -2.0), np.ones(o.nnz)
    o.set_system(d, lu, np.ones(o.n))
    lv = o.amg_levels()
    assert lv[1]["n"] == 3
    assert lv[1]["agg"].tolist() == [0, 0, 1, 1, 1, 2, 2, 2]
    assert heap_aggregation([[1]] + [[i - 1, i + 1] for i in range(1, 7)] + [[6]]) == [0, 0, 1, 1, 1, 2, 2, 2]
    o.close()


@pytest.mark.parametrize("shape,seed", [((12, 10, 8), 4), ((20, 16, 10), 7)])
def test_heap_matches_second_restatement(shape, seed):
    """The oracle's heap aggregation equals the dict-based restatement node for node on the
    fine-level strength graph of a heterogeneous block."""
    p, o, d, lu, r = _system(shape, seed)
    o.set_aggregation(1)
    o.set_system(d, lu, r)
    lv = o.amg_levels()
    strong = _strength(d, lu, lv[0]["offind"], lv[0]["offrow"], p.params["amg_theta"])
    want = heap_aggregation(strong)
    assert lv[1]["agg"].tolist() == want
    assert lv[1]["n"] == max(want) + 1
    o.close()


def test_heap_against_mis2_structure():
    """The reference's aggregation and the MIS-2 on the same Jacobians: both coarsen by
    a similar ratio; the heap leaves its distance-2 rings out of every aggregate (they are
    reached only through the smoothed prolongation) where MIS-2 places every node with a
    strong connection; both V-cycles make BiCGStab converge."""
    rows = []
    for shape, seed in (((24, 20, 16), 6), ((40, 36, 20), 8)):
        p, o, d, lu, r = _system(shape, seed)
        res = {}
        for mode in (0, 1):
            o.set_aggregation(mode)
            o.set_system(d, lu, r)
            lv = o.amg_levels()
            agg = lv[1]["agg"]
            strong = _strength(d, lu, lv[0]["offind"], lv[0]["offrow"], p.params["amg_theta"])
            strong_rows = np.array([len(row) > 0 for row in strong])
            _, last, it, conv = o.solve_linalg(float(np.sqrt(np.sum(r * r))), 1e-8)
            res[mode] = dict(levels=[l["n"] for l in lv], out=float(np.mean(agg[strong_rows] < 0)),
                             nnz_row=len(lv[1]["offrow"]) / lv[1]["n"], iters=it, conv=conv)
        rows.append((shape, res))
        print(f"{shape}: MIS-2 {res[0]}\n{'':>14} heap  {res[1]}")
        assert res[0]["conv"] == 1 and res[1]["conv"] == 1
        assert res[0]["out"] == 0.0 and res[1]["out"] > 0.0
        ratio0 = res[0]["levels"][0] / res[0]["levels"][1]
        ratio1 = res[1]["levels"][0] / res[1]["levels"][1]
        assert 0.25 < ratio1 / ratio0 < 4.0
        o.close()
