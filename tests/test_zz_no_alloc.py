"""claw_step2d_noalloc: the step entry point that allocates no device memory.

Callers that own all their device memory (a framework's caching allocator, a
fixed-budget coupled model) hand the library their own q_in / q_out buffers;
the step kernel's scratch then comes from a static device array instead of
cudaMalloc.  This test drives that entry point through the C ABI on buffers
owned by the caller (torch here) and checks two calls in a row against the
regular handle-based claw_step, bit for bit (the tolerance of every FP64
parity test in this suite).  It runs last (file name) so that a failure here
leaves the rest of the suite already run, and it needs no state from earlier
tests."""
import ctypes

import numpy as np
import pytest

from classic_b200 import _lib, problems
from classic_b200.solver import Solver, make_config

pytestmark = pytest.mark.gpu


def _cases():
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=256)
    yield "mc-specialised", rd, solver, params, q0, None
    rd, solver, params, q0, _ = problems.random_acoustics_2d(
        57, 40, seed=5, limiter="vanleer", bc=("wall", "periodic", "periodic", "wall"))
    rd.clawdata.bc_lower = ["wall", "periodic"]
    rd.clawdata.bc_upper = ["wall", "periodic"]
    yield "generic", rd, solver, params, q0, None
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    yield "capacity+aux", rd, solver, params, q0, aux


@pytest.mark.parametrize("case", ["mc-specialised", "generic", "capacity+aux"])
def test_noalloc_matches_claw_step_twice(case):
    import torch

    name, rd, solver, params, q0, aux = next(c for c in _cases() if c[0] == case)
    lib = _lib.load()
    cd = rd.clawdata
    mx, my = cd.num_cells
    meqn = cd.num_eqn
    dt_list = [0.8 * min(2.0 / mx, 2.0 / my) / 2.0, 0.7 * min(2.0 / mx, 2.0 / my) / 2.0]
    if solver == "vc_advection_2d":
        dt_list = [0.002, 0.0015]

    # regular path: handle-owned memory
    ref = Solver(cd, solver, params)
    ref.set_q(q0)
    if aux is not None:
        ref.set_aux(aux)
    expected = []
    for dt in dt_list:
        c = ref.step(dt)
        expected.append((ref.get_q(), c))
    ref.close()

    # caller-owned device buffers (row pitch padded to an even count)
    ld = mx + (mx % 2)
    dev = torch.device("cuda", 0)
    bufs = [torch.zeros((meqn, my, ld), dtype=torch.float64, device=dev) for _ in range(2)]
    bufs[0][:, :, :mx] = torch.from_numpy(np.ascontiguousarray(q0)).to(dev)
    aux_t, aux_ld = None, 0
    if aux is not None:
        aux_ld = (mx + 4) + ((mx + 4) % 2)
        aux_t = torch.zeros((aux.shape[0], my + 4, aux_ld), dtype=torch.float64, device=dev)
        aux_t[:, :, : mx + 4] = torch.from_numpy(np.ascontiguousarray(aux)).to(dev)
    cfg = make_config(cd, solver, params)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    src, dst = 0, 1
    for k, dt in enumerate(dt_list):
        cfl = ctypes.c_double(-1.0)
        rc = lib.claw_step2d_noalloc(ctypes.byref(cfg), ctypes.c_void_p(bufs[src].data_ptr()),
                                     ctypes.c_void_p(bufs[dst].data_ptr()), ld,
                                     ctypes.c_void_p(aux_t.data_ptr() if aux_t is not None else 0),
                                     aux_ld, dt, ctypes.byref(cfl), stream)
        assert rc == 0, lib.claw_last_error().decode()
        got = bufs[dst][:, :, :mx].cpu().numpy()
        want_q, want_cfl = expected[k]
        assert cfl.value == want_cfl
        assert np.array_equal(got, want_q), f"{name}: call {k + 1} differs"
        src, dst = dst, src


def test_noalloc_rejects_bad_requests():
    lib = _lib.load()
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=64)
    cfg = make_config(rd.clawdata, solver, params, precision="fp32")
    cfl = ctypes.c_double(0.0)
    # FP32 is not served by this entry point; nothing is launched
    rc = lib.claw_step2d_noalloc(ctypes.byref(cfg), ctypes.c_void_p(16), ctypes.c_void_p(32), 64,
                                 None, 0, 0.001, ctypes.byref(cfl), None)
    assert rc == -1
    cfg = make_config(rd.clawdata, solver, params)
    rc = lib.claw_step2d_noalloc(ctypes.byref(cfg), ctypes.c_void_p(16), ctypes.c_void_p(16), 64,
                                 None, 0, 0.001, ctypes.byref(cfl), None)
    assert rc == -1  # q_in == q_out
    rc = lib.claw_step2d_noalloc(ctypes.byref(cfg), ctypes.c_void_p(16), ctypes.c_void_p(32), 63,
                                 None, 0, 0.001, ctypes.byref(cfl), None)
    assert rc == -1  # odd row pitch
    # a before-step routine needs a copy of the unscaled aux this path cannot allocate
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    cfg = make_config(rd.clawdata, solver, params)
    cfg.b4step_id = 1
    cfg.b4step_param = 1.0
    rc = lib.claw_step2d_noalloc(ctypes.byref(cfg), ctypes.c_void_p(16), ctypes.c_void_p(32), 64,
                                 ctypes.c_void_p(64), 68, 0.001, ctypes.byref(cfl), None)
    assert rc == -3


def test_noalloc_refuses_stream_capture():
    """A captured graph could not replay the call's stream wait and host upload:
    the entry point refuses before touching the stream."""
    import torch

    lib = _lib.load()
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=64)
    cfg = make_config(rd.clawdata, solver, params)
    dev = torch.device("cuda", 0)
    bufs = [torch.zeros((3, 64, 64), dtype=torch.float64, device=dev) for _ in range(2)]
    cfl = ctypes.c_double(0.0)
    side = torch.cuda.Stream(dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        rc = lib.claw_step2d_noalloc(ctypes.byref(cfg), ctypes.c_void_p(bufs[0].data_ptr()),
                                     ctypes.c_void_p(bufs[1].data_ptr()), 64, None, 0, 0.001,
                                     ctypes.byref(cfl), ctypes.c_void_p(side.cuda_stream))
        bufs[1].add_(1.0)
    assert rc == -1
    assert "capture" in lib.claw_last_error().decode()
    del graph
