"""dic_cuda_solve_noalloc against dic_cuda_solve.

dic_cuda_solve_noalloc is for callers that cannot allocate device memory:
code running inside a host application that owns the device-memory pool, or
under a fixed memory budget, where a cudaMalloc for scratch is not allowed.
It keeps the solve's scratch in a fixed array inside the library, so the
caller passes only inputs and outputs. These tests call it through the C ABI
and require the same results, bit for bit (the tolerance of every solve
test here), as the allocating entry point, on two calls in a row: the second
call must not see anything the first one left in the shared array.

The file name sorts last, so a run that stops at the first failure has run
every other test before this one.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import semper_b200 as sb

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _header_max_tasks():
    h = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "semper_dic_cuda.h")
    m = re.search(r"#define\s+DIC_CUDA_SOLVE_NOALLOC_MAX_TASKS\s+(\d+)", open(h).read())
    return int(m.group(1))


MAX_TASKS = _header_max_tasks()  # read from the header the library is built from
CUDA_ERROR_INVALID_VALUE = 1


def _noalloc():
    f = sb.lib().dic_cuda_solve_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp] * 4 + [ctypes.c_int] * 3 + [vp] * 3 + [ctypes.c_int] * 3 + [vp, ctypes.c_int, vp,
                                                                                       ctypes.c_int, vp]
    f.restype = ctypes.c_int
    return f


def _case(n, seed, warp, noise, mask, xy, guess, mode, subset, six):
    ref = sb.speckle(n, n, seed)
    dfm = sb.speckle(n, n, seed, warp, 1.0, noise)
    rplanes = sb.image_prep(torch.from_numpy(ref).cuda(), None if mask is None else torch.from_numpy(mask).cuda())
    dI = sb.image_prep(torch.from_numpy(dfm).cuda())[0]
    k = len(xy)
    valid = torch.zeros(k, dtype=torch.uint8, device="cuda")
    ms = torch.zeros((k, 2), dtype=torch.float32, device="cuda")
    Hs = torch.zeros((k, 21), dtype=torch.float64, device="cuda")
    for i, (x, y) in enumerate(xy):
        sk = torch.zeros(1, dtype=torch.uint8, device="cuda")
        v1, m1, _h1, hs1 = sb.hessian_pool(rplanes, n, sk, (1, 1), (int(x), int(y)), 1, subset, True)
        valid[i], ms[i], Hs[i] = v1[0], m1[0], hs1[0]
    tasks = np.zeros(k, sb.TASK_DT)
    tasks["node"] = np.arange(k)
    tasks["cx"], tasks["cy"] = xy[:, 0], xy[:, 1]
    tasks["mode"] = mode
    tasks["g"] = guess
    return rplanes, dI, (valid, ms, None, Hs), tasks


def _run_noalloc(rplanes, dI, width, pool, subset, tasks, six):
    rI, rgx, rgy = rplanes
    valid, ms, _h, Hs = pool
    n = len(tasks)
    tb = torch.from_numpy(np.ascontiguousarray(tasks).view(np.uint8).copy()).cuda()
    res = torch.zeros(n * sb.RESULT_DT.itemsize, dtype=torch.uint8, device="cuda")
    rc = _noalloc()(rI.data_ptr(), rgx.data_ptr(), rgy.data_ptr(), dI.data_ptr(), width, rI.shape[0], rI.shape[1],
                    valid.data_ptr(), ms.data_ptr(), Hs.data_ptr(), subset, 1, 1 if six else 0, tb.data_ptr(), n,
                    res.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    return res.cpu().numpy().view(sb.RESULT_DT).copy()


def _cases():
    n = 256
    rng = np.random.default_rng(3)
    xy = rng.integers(20, n - 20, size=(64, 2)).astype(np.int32)
    far = np.zeros((64, 6), np.float32)
    far[:, 0], far[:, 1] = 1.0, -0.5
    far[::5, 0] = 6.0  # far guesses: Simplex rescues, handed on to the general pass
    warp = sb.warp_block(cx=128, cy=128, u0=1.3, v0=-0.7, a=(0.01, -0.004, 0.003, -0.006))
    yield "rescue", (n, 5, warp, 77, None, xy, far, sb.INIT_NO_SEARCH, 21, False)
    yield "search", (n, 5, warp, 77, None, xy, np.zeros((64, 6), np.float32), sb.INIT_AUTO_SEARCH, 21, True)
    m = 200
    yy, xx = np.mgrid[0:m, 0:m]
    mask = np.full((m, m), 255, np.uint8)
    mask[(xx - 100) ** 2 + (yy - 100) ** 2 < 25 * 25] = 0
    grid = np.array([(x, y) for y in range(16, m - 10, 11) for x in range(16, m - 10, 11)], np.int32)
    g = np.tile(np.array([2.0, 1.0, 0, 0, 0, 0], np.float32), (len(grid), 1))
    yield "masked", (m, 9, sb.warp_block(u0=2.2, v0=1.1), 5, mask, grid, g, sb.INIT_NO_SEARCH, 25, False)


@pytest.mark.parametrize("name,args", list(_cases()), ids=[c[0] for c in _cases()])
def test_noalloc_matches_allocating_solve_twice(name, args):
    n, subset, six = args[0], args[8], args[9]
    rplanes, dI, pool, tasks = _case(*args)
    want = sb.solve(rplanes, dI, n, pool, subset, tasks, lm=True, six=six)
    assert (want["flags"] & 1).sum() > len(tasks) // 2
    for _ in range(2):
        got = _run_noalloc(rplanes, dI, n, pool, subset, tasks, six)
        assert got.tobytes() == want.tobytes()


def test_noalloc_rejects_more_tasks_than_its_scratch_holds():
    # checked before any device work: no pointer is touched
    rc = _noalloc()(None, None, None, None, 64, 64, 64, None, None, None, 21, 1, 0, None, MAX_TASKS + 1, None, 0,
                    None)
    assert rc == CUDA_ERROR_INVALID_VALUE


def test_noalloc_accepts_exactly_the_maximum_task_count():
    """MAX_TASKS tasks fill the fixed scratch exactly: the call is accepted and
    solves them as dic_cuda_solve does. The tasks repeat 64 subsets of a small
    pair (pool rows = task index, tiled on the device)."""
    args = dict(_cases())["rescue"]
    n, subset = args[0], args[8]
    rplanes, dI, (valid, ms, _h, Hs), tasks = _case(*args)
    reps = MAX_TASKS // len(tasks)
    assert reps * len(tasks) == MAX_TASKS
    big = np.tile(tasks, reps)
    big["node"] = np.arange(MAX_TASKS)
    pool = (valid.repeat(reps), ms.repeat(reps, 1), None, Hs.repeat(reps, 1))
    want = sb.solve(rplanes, dI, n, pool, subset, big, lm=True, six=False)
    got = _run_noalloc(rplanes, dI, n, pool, subset, big, False)
    assert got.tobytes() == want.tobytes()
