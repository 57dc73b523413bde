"""The C-ABI library loads without a GPU and exports every function that
include/matvans.h declares."""
import ctypes
import os
import re

from conftest import ROOT
from matvans_b200 import _lib


def declared_functions():
    src = open(os.path.join(ROOT, "include", "matvans.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"if", "for", "while", "return", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip and (n.startswith("mv_") or n.startswith("mat_vec_mul_coalesced"))})


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    decl = declared_functions()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == decl


def test_version_and_error_string():
    L = _lib.lib()
    assert b"sm_100a" in L.mv_version()
    rc = L.mv_awr_encode(None, 0, 0, 0, ctypes.byref(ctypes.c_void_p()))
    assert rc == 1
    assert b"bad arguments" in L.mv_last_error()


def test_stack_plan_reports_atomic_jobs():
    """The stack plan counts the jobs whose rows span several work items (parts > 1 and more than one
    segment): only then does the launch add its zero and scale passes.  Host only."""
    from matvans_b200._lib import Q8Job, Q8StackInfo, Q8Tuning
    L = _lib.lib()
    jobs = (Q8Job * 3)()
    for i, (r, c) in enumerate([(64, 512), (32, 64), (96, 1024)]):
        jobs[i].m.rows, jobs[i].m.cols = r, c
        jobs[i].m.seg_quads = 16
        jobs[i].m.nseg = -(-(c // 4) // 16)
        jobs[i].m.local = 1
        jobs[i].m.max_blk_rows = 4
    info = Q8StackInfo()
    assert L.mv_q8_stack_plan(jobs, 3, ctypes.byref(Q8Tuning(8, 1, 1, 0, 0, 0)), ctypes.byref(info)) == 0
    assert info.atomic_jobs == 0 and all(jobs[i].atomic == 0 for i in range(3))
    assert info.nitems == 2 + 1 + 3
    # the plan orders the jobs by work per item, most first (whole stripes: by columns), and numbers the
    # items job by job in that order
    assert [jobs[i].m.cols for i in range(3)] == [1024, 512, 64]
    assert [jobs[i].item0 for i in range(3)] == [0, 3, 5]
    # parts = 4: every job with more than one segment is split (and accumulates atomically); the
    # 64-column job has a single segment and stays whole
    assert L.mv_q8_stack_plan(jobs, 3, ctypes.byref(Q8Tuning(8, 1, 1, 0, 4, 0)), ctypes.byref(info)) == 0
    by_cols = {jobs[i].m.cols: jobs[i] for i in range(3)}
    assert [by_cols[c].ngroups for c in (512, 64, 1024)] == [4, 1, 4]
    assert info.atomic_jobs == 2 and [by_cols[c].atomic for c in (512, 64, 1024)] == [1, 0, 1]
    assert info.nitems == 2 * 4 + 1 + 3 * 4


def test_tensor_core_threshold_matches_the_header():
    """The Python side's batch threshold for the tensor-core engine (ops, autotuner, bench) is the library's."""
    src = open(os.path.join(ROOT, "include", "matvans.h")).read()
    m = re.search(r"#define\s+MV_MMA_MIN_VECTORS\s+(\d+)", src)
    assert m and int(m.group(1)) == _lib.MMA_MIN_BATCH
