"""Trace export on the host (no GPU): the tables carry the column layout of
the reference's trace converter (bin/ukilli.cpp:887-889, 916-918, 934-936,
952-954, 966-971), argument errors are reported, and API calls are recorded
as host tasks and closed by xkblas_sync."""
import csv
import ctypes
import errno
import os

import numpy as np
import pytest

import xkblas_b200 as X

HEADERS = {
    "kern.csv": "Resource,Type,Stream,Push,Start,End,Duration,Name,TaskId",
    "cpy.csv": "Resource,Type,Stream,Push,Start,End,Duration,Size,Dir",
    "task.csv": "Resource,Type,Push,Start,End,Duration,Name,TaskId",
    "parallel.csv": "Resource,Type,Start,End,Duration,Name",
    "call.csv": "Resource,Level,Start,End,Duration,Name,NParam,"
                + ",".join("Param%d" % i for i in range(16)),
}


def _rows(path):
    with open(path, newline="") as f:
        return list(csv.DictReader(f))


@pytest.fixture
def lib():
    L = X.lib()
    L.xkblas_trace_record(0)
    yield L
    L.xkblas_trace_record(0)


def test_headers_without_events(lib, tmp_path):
    assert lib.xkblas_trace_export(os.fsencode(str(tmp_path))) == 0
    for name, header in HEADERS.items():
        with open(tmp_path / name) as f:
            assert f.readline().rstrip("\n") == header, name


def test_export_errors(lib, tmp_path):
    assert lib.xkblas_trace_export(None) == errno.EINVAL
    assert lib.xkblas_trace_export(b"") == errno.EINVAL
    assert lib.xkblas_trace_export(os.fsencode(str(tmp_path / "no" / "such"))) == errno.EIO


def test_record_toggle(lib):
    assert lib.xkblas_trace_record(1) == 0
    assert lib.xkblas_trace_record(1) == 1
    assert lib.xkblas_trace_record(0) == 1
    assert lib.xkblas_trace_record(0) == 0


def test_call_recorded_and_closed_by_sync(lib, tmp_path):
    if X.lib().xkblas_get_devicecount() > 0:
        pytest.skip("host-only case: with a GPU the call runs (covered by test_gpu_trace)")
    lib.xkblas_trace_export(os.fsencode(str(tmp_path)))  # drain earlier events
    lib.xkblas_trace_record(1)
    a = np.ones((3, 3), order="F")
    one = np.ones(1)
    p = lambda v: ctypes.c_void_p(v.ctypes.data)
    # no device here: the call fails, but it was made and is traced
    assert lib.xkblas_dgemm_async(111, 112, 3, 2, 3, p(one), p(a), 3, p(a), 3, p(one), p(a), 3) != 0
    assert lib.xkblas_sync() == 0
    out = tmp_path / "t"
    out.mkdir()
    assert lib.xkblas_trace_export(os.fsencode(str(out))) == 0
    tasks = _rows(out / "task.csv")
    calls = _rows(out / "call.csv")
    assert [t["Name"] for t in tasks] == ["dgemm"]
    assert len(calls) == 1
    c = calls[0]
    assert c["Name"] == "dgemm" and c["NParam"] == "7" and c["Level"] == "0"
    assert (c["Param0"], c["Param1"], c["Param2"]) == ("3", "2", "3")
    assert (c["Param4"], c["Param5"]) == ("111", "112")
    assert float(c["End"]) >= float(c["Start"]) >= 0.0
    assert abs(float(c["Duration"]) - (float(c["End"]) - float(c["Start"]))) < 1e-9
    assert _rows(out / "kern.csv") == [] and _rows(out / "cpy.csv") == []
    # exported events leave the log
    again = tmp_path / "u"
    again.mkdir()
    assert lib.xkblas_trace_export(os.fsencode(str(again))) == 0
    assert _rows(again / "task.csv") == [] and _rows(again / "call.csv") == []


def test_calls_from_two_threads(lib, tmp_path):
    """Each host thread is its own CPU resource (the reference's kproc id) and
    its xkblas_sync closes only its own calls (ukilli.cpp:762-775)."""
    import threading
    if X.lib().xkblas_get_devicecount() > 0:
        pytest.skip("host-only case")
    lib.xkblas_trace_export(os.fsencode(str(tmp_path)))  # drain earlier events
    lib.xkblas_trace_record(1)
    a = np.ones((4, 4), order="F")
    one = np.ones(1)
    p = lambda v: ctypes.c_void_p(v.ctypes.data)
    barrier = threading.Barrier(2)

    def work(n_calls, do_sync):
        barrier.wait()
        for _ in range(n_calls):
            lib.xkblas_dtrsm_async(141, 122, 111, 131, 4, 4, p(one), p(a), 4, p(a), 4)
        if do_sync:
            assert lib.xkblas_sync() == 0

    t1 = threading.Thread(target=work, args=(3, True))
    t2 = threading.Thread(target=work, args=(2, False))
    t1.start(); t2.start(); t1.join(); t2.join()
    out = tmp_path / "t2"
    out.mkdir()
    assert lib.xkblas_trace_export(os.fsencode(str(out))) == 0
    tasks = _rows(out / "task.csv")
    calls = _rows(out / "call.csv")
    by_res = {}
    for t in tasks:
        by_res.setdefault(t["Resource"], []).append(t["Name"])
    assert sorted(len(v) for v in by_res.values()) == [2, 3]
    assert all(n == "dtrsm" for v in by_res.values() for n in v)
    # only the syncing thread's three calls are closed, at levels 0..2
    assert len(calls) == 3
    assert sorted(c["Level"] for c in calls) == ["0", "1", "2"]
    assert len({c["Resource"] for c in calls}) == 1
    assert [int(calls[0]["Param%d" % i]) for i in range(6)] == [4, 4, 141, 122, 111, 131]
    # the other thread's calls stay open until its own sync
    lib.xkblas_trace_record(0)
