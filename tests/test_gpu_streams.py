"""The table build forks its (la, lb) groups and its per-class record kernels
onto side streams and joins them back into the caller's stream.  A build on a
non-default stream, and builds issued from two host threads on two streams at
once, give the same table, bit for bit, as a build on the default stream."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from fastesp_b200 import build_table

pytestmark = pytest.mark.gpu


def _arrays(tab):
    return [tab.records(L).copy() for L, c in enumerate(tab.counts) if c]


def test_build_on_a_side_stream(frag54, golden):
    import torch
    wfn, basis, P = frag54
    g = golden("frag54_300")
    ref = build_table(wfn, basis, P, g["points"], tol=1e-12)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        tab = build_table(wfn, basis, P, g["points"], tol=1e-12)
        v = tab.esp(g["points"])
    s.synchronize()
    assert tab.counts == ref.counts
    for a, b in zip(_arrays(tab), _arrays(ref)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(v, ref.esp(g["points"]))


def test_builds_from_two_threads(frag54, golden):
    import torch
    wfn, basis, P = frag54
    g = golden("frag54_300")
    ref = build_table(wfn, basis, P, g["points"], tol=1e-12)
    want = ref.esp(g["points"])
    out, errs = [None, None], []

    def work(i):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                t = build_table(wfn, basis, P, g["points"], tol=1e-12)
                out[i] = (t.counts, t.esp(g["points"]))
            s.synchronize()
        except Exception as e:          # reported below, in the main thread
            errs.append(e)
    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for counts, v in out:
        assert counts == ref.counts
        np.testing.assert_array_equal(v, want)
