"""Right-hand side through shhd_rhs_noalloc, the entry point that allocates no device memory (GPU).

Some hosts cannot call cudaMalloc: a solver embedded in a framework whose
caching allocator owns the GPU's memory, or a plugin in a process that
reserved its device memory up front.  shhd_rhs_noalloc serves them: the caller
passes device buffers it already owns, and every intermediate lives in a
fixed array compiled into the library.  These tests call it through the C ABI
and check it against shhd_engine_rhs (the engine entry point, which allocates)
and against the FP64 oracle's right-hand side, on consecutive calls, so that
anything left in the shared array by one call would show up in the next.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5

CASES = [
    # compile-time transform sizes (64 -> 96), compressible, phi4 + advection
    dict(grid=(64, 64), length=(64.0, 64.0), nop=2, dt=0.01),
    # runtime-plan sizes (40 x 36 -> 60 x 54), compressible
    dict(grid=(40, 36), length=(40.0, 30.0), nop=1, dt=0.01),
    # incompressible: uses the reference density of the input state
    dict(grid=(64, 64), length=(64.0, 64.0), nop=0, dt=0.01, te="srk3/incompressible", cT=None, eta=0.05, zeta=0.0,
         nonlinear="momentum"),
    # quiescent: psi only, the physical chemical potential is the one product
    dict(grid=(64, 64), length=(128.0, 128.0), nop=1, dt=0.02, te="srk3/quiescent", cT=None, eta=0.0, zeta=0.0, nonlinear=None),
]


def _noalloc(sb, torch, cfg, state, stream=None):
    """Upload `state`, call shhd_rhs_noalloc on caller-owned device buffers, return the RHS."""
    flat = np.ascontiguousarray(state, dtype=np.complex128).view(np.float64).ravel()
    dev_in = torch.from_numpy(flat.copy()).to("cuda")
    dev_out = torch.full_like(dev_in, float("nan"))  # every entry must be written
    torch.cuda.synchronize()
    c = cfg.copy()
    rc = sb.lib.shhd_rhs_noalloc(ctypes.byref(c), ctypes.c_void_p(dev_in.data_ptr()), ctypes.c_void_p(dev_out.data_ptr()),
                                 flat.size, ctypes.c_void_p(stream))
    if rc != sb.SHHD_OK:
        raise sb.ShhdError(rc, sb.lib.shhd_last_error().decode())
    return dev_out.cpu().numpy().view(np.complex128).reshape(state.shape)


def _engine_rhs(sb, cfg, state):
    with sb.Engine(cfg) as eng:
        eng.set_state(state)
        return eng.rhs()


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_rhs_matches_engine_on_consecutive_calls(precision):
    import torch
    import shhd_b200 as sb
    tol = TOL64 if precision == 0 else TOL32
    for ci, kw in enumerate(CASES):
        text = script(**kw)
        cfg = sb.config_from_script(text)
        cfg.precision = precision
        ocfg = so.parse_script(text)
        transverse = ocfg.mode == "incompressible"
        # two calls in a row on one configuration (different states, different densities),
        # then the next configuration follows on the same shared scratch
        for call, seed in enumerate((11 + ci, 23 + ci)):
            u = random_state(ocfg, seed=seed, rho0=1.0 + 0.25 * call, transverse=transverse)
            want = _engine_rhs(sb, cfg, u)
            got = _noalloc(sb, torch, cfg, u)
            assert np.all(np.isfinite(got))
            err = so.rel_l2(got, want)
            assert err < tol, f"case {ci} call {call}: rel L2 {err:.3e}"


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_rhs_matches_oracle(precision):
    """The same calls against the FP64 oracle's deterministic RHS directly (not only the engine)."""
    import torch
    import shhd_b200 as sb
    tol = TOL64 if precision == 0 else TOL32
    for ci, kw in enumerate(CASES):
        text = script(**kw)
        cfg = sb.config_from_script(text)
        cfg.precision = precision
        ocfg = so.parse_script(text)
        for call, seed in enumerate((41 + ci, 53 + ci)):
            u = random_state(ocfg, seed=seed, rho0=1.0 + 0.5 * call, transverse=ocfg.mode == "incompressible")
            want = so.Oracle(ocfg).rhs(u)
            got = _noalloc(sb, torch, cfg, u)
            err = so.rel_l2(got, want)
            assert err < tol, f"case {ci} call {call}: rel L2 {err:.3e} against the oracle"


def test_noalloc_rhs_on_a_caller_stream():
    import torch
    import shhd_b200 as sb
    text = script(**CASES[0])
    cfg = sb.config_from_script(text)
    u = random_state(so.parse_script(text), seed=5)
    want = _engine_rhs(sb, cfg, u)
    s = torch.cuda.Stream()
    for _ in range(2):
        got = _noalloc(sb, torch, cfg, u, stream=s.cuda_stream)
        assert so.rel_l2(got, want) < TOL64


def test_noalloc_rejects_what_it_cannot_hold():
    import torch
    import shhd_b200 as sb
    # 1024^2 with 3/2 padding and two order parameters needs far more than the static scratch
    text = script(grid=(1024, 1024), length=(1024.0, 1024.0), nop=2, dt=0.01)
    cfg = sb.config_from_script(text)
    n = 5 * 1536 * (1536 // 2 + 1) * 2
    a = torch.zeros(n, dtype=torch.float64, device="cuda")
    b = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc = sb.lib.shhd_rhs_noalloc(ctypes.byref(cfg), ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), n, None)
    assert rc == sb.SHHD_EINVAL
    msg = sb.lib.shhd_last_error().decode()
    assert "static scratch holds" in msg and "bytes" in msg
    # host memory is refused before any work is enqueued
    small = script(**CASES[0])
    c2 = sb.config_from_script(small)
    u = np.ascontiguousarray(random_state(so.parse_script(small), seed=1)).view(np.float64).ravel()
    out = np.zeros_like(u)
    rc = sb.lib.shhd_rhs_noalloc(ctypes.byref(c2), u.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p), u.size, None)
    assert rc == sb.SHHD_EINVAL
    assert "device memory" in sb.lib.shhd_last_error().decode() or "CUDA pointer" in sb.lib.shhd_last_error().decode()


@pytest.mark.filterwarnings("ignore:The CUDA Graph is empty")
def test_noalloc_refuses_a_capturing_stream():
    """The call is synchronous: on a stream under graph capture it returns SHHD_EINVAL before
    enqueuing anything, and the capture ends normally."""
    import torch
    import shhd_b200 as sb
    text = script(**CASES[0])
    cfg = sb.config_from_script(text)
    state = random_state(so.parse_script(text), seed=71)
    flat = np.ascontiguousarray(state, dtype=np.complex128).view(np.float64).ravel()
    dev_in = torch.from_numpy(flat.copy()).to("cuda")
    dev_out = torch.zeros_like(dev_in)
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    c = cfg.copy()
    with torch.cuda.graph(graph, stream=side):
        rc = sb.lib.shhd_rhs_noalloc(ctypes.byref(c), ctypes.c_void_p(dev_in.data_ptr()), ctypes.c_void_p(dev_out.data_ptr()),
                                     flat.size, ctypes.c_void_p(side.cuda_stream))
    assert rc == sb.SHHD_EINVAL
    assert "cannot run on a stream that is being captured" in sb.lib.shhd_last_error().decode()
    del graph
    # the entry point still works afterwards
    got = _noalloc(sb, torch, cfg, state)
    assert so.rel_l2(got, so.Oracle(so.parse_script(text)).rhs(state)) < TOL64
