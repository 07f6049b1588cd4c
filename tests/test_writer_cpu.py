"""Result files written by the library (host.cpp write_result behind
qc_sets_write_async): the reference's line format "<k> v1 .. vk \\n"
(main.cu:4641-4652), large outputs formatted in parallel chunks and written in
order, writes that overlap the caller, and malformed input rejected."""
import os
import tempfile

import numpy as np
import pytest

import cuqc_b200 as Q


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(Q.LIB_PATH):
        Q.build()


def reference_text(sets):
    return "".join("%d " % len(s) + "".join("%d " % v for v in s) + "\n" for s in sets)


def flat_of(sets):
    out = []
    for s in sets:
        out.append(len(s))
        out.extend(s)
    return np.asarray(out, np.int32)


def test_small_result_text():
    sets = [(0, 1, 2), (3,), (4, 10, 2000000000)]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "r.txt")
        Q.write_sets_async(flat_of(sets), p).wait()
        assert open(p).read() == reference_text(sets)


def test_empty_result_writes_an_empty_file():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "r.txt")
        Q.write_sets_async(np.zeros(0, np.int32), p).wait()
        assert os.path.getsize(p) == 0


def test_large_result_in_parallel_chunks_keeps_order():
    rng = np.random.default_rng(7)
    sets = [tuple(sorted(rng.choice(10 ** 6, size=int(rng.integers(5, 40)), replace=False).tolist()))
            for _ in range(60000)]  # about 1.3 M ints: several chunks
    flat = flat_of(sets)
    with tempfile.TemporaryDirectory() as d:
        ps = [os.path.join(d, "r%d.txt" % i) for i in range(3)]
        ws = [Q.write_sets_async(flat, p) for p in ps]  # three writes at once
        for w in ws:
            w.wait()
        want = reference_text(sets)
        for p in ps:
            assert open(p).read() == want


def test_result_object_writes():
    sets = [(1, 2, 3), (2, 5)]
    r = Q.Result(flat_of(sets), {})
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "r.txt")
        r.write(p)
        assert open(p).read() == reference_text(sets)
        w = r.write_async(p + "2")
        w.wait()
        assert open(p + "2").read() == reference_text(sets)


def test_malformed_and_unwritable():
    with tempfile.TemporaryDirectory() as d:
        with pytest.raises(Q.QCError) as e:
            Q.write_sets_async(np.asarray([3, 1, 2], np.int32), os.path.join(d, "r.txt")).wait()
        assert Q.STATUS[e.value.status] == "QC_ERR_FORMAT"
        with pytest.raises(Q.QCError) as e:
            Q.write_sets_async(np.asarray([1, 1], np.int32), os.path.join(d, "no", "r.txt")).wait()
        assert Q.STATUS[e.value.status] == "QC_ERR_IO"
