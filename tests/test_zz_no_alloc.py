"""scarl_gen_padded_noalloc: the generator for callers that cannot allocate
GPU memory (their device memory belongs to their own pool allocator, or they
run a loop that must not call cudaMalloc).  Checked through the C ABI against
the allocating entry point scarl_gen_padded, on two calls in a row that share
the fixed scratch array.  Collected last, so a failure here stops a -x run
only after every other test has run."""
import ctypes as C

import numpy as np
import pytest

import scarl_b200 as S
from scarl_b200 import _lib

pytestmark = pytest.mark.gpu


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _noalloc(out, Np, pad, dx, cl, cm, nu, seed, stream, dtype=S.F32, normalise=1):
    msg = C.create_string_buffer(256)
    rc = _lib.lib().scarl_gen_padded_noalloc(C.c_void_p(out.data_ptr()), dtype, _i3(Np),
                                             _i3(pad) if pad else None, _d3(dx), _d3(cl), cm, nu,
                                             normalise, seed, stream, None, msg, 256)
    return rc, msg.value.decode()


CASES = [  # Np, pad, xStep, corrL, corrMod, nu, seed, stream, normalise
    ((60, 50, 40), (128, 128, 128), (1.0, 1.0, 1.0), (8.0, 6.0, 5.0), 3, 0.5, 11, 0, 1),
    ((100, 33, 70), (256, 64, 128), (0.5, 1.0, 1.0), (9.0, 4.0, 7.0), 1, 0.5, 12345, 3, 1),
    # von Karman nu = 1.5: the power-law amplitude tables
    ((40, 30, 50), (64, 64, 128), (1.0, 1.0, 1.0), (6.0, 5.0, 9.0), 2, 1.5, 7, 1, 1),
    # no spectral normalisation (no host wait), default padded grid 64 x 32 x 64
    ((20, 16, 30), None, (1.0, 1.0, 1.0), (4.0, 3.0, 5.0), 3, 0.5, 99, 2, 0),
    # mixed-radix padded lengths 320 = 5 x 64, 192 = 3 x 64, 112 = 7 x 16
    ((90, 70, 60), (320, 192, 112), (1.0, 1.0, 1.0), (7.0, 6.0, 5.0), 3, 0.5, 5, 0, 1),
]


@pytest.mark.parametrize("dtype,tol", [(S.F32, 1e-6), (S.F64, 1e-13)])
def test_noalloc_matches_allocating_entry_point_twice(ctx, dtype, tol):
    """Each case runs twice in a row through the shared scratch array and
    matches scarl_gen_padded; the GPU's free memory is the same before and
    after all the calls."""
    torch = pytest.importorskip("torch")
    tdt = torch.float32 if dtype == S.F32 else torch.float64
    refs, outs = [], []
    for Np, pad, dx, cl, cm, nu, seed, stream, nrm in CASES:
        refs.append(S.gen_padded(ctx, Np, dx, cl, cm, nu, pad=pad, normalise=bool(nrm), seed=seed,
                                 stream=stream, dtype=dtype))
        outs.append([torch.full((int(np.prod(Np)),), float("nan"), dtype=tdt, device="cuda")
                     for _ in range(2)])
    # a first call: the scratch array's module may load (and reserve its
    # 64 MiB) when its address is first looked up
    warm = torch.empty(64, dtype=tdt, device="cuda")  # 4^3 points, default grid 8^3
    assert _noalloc(warm, (4, 4, 4), None, (1, 1, 1), (1, 1, 1), 1, 0.5, 0, 0, dtype)[0] == _lib.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for (Np, pad, dx, cl, cm, nu, seed, stream, nrm), pair in zip(CASES, outs):
        for out in pair:
            rc, msg = _noalloc(out, Np, pad, dx, cl, cm, nu, seed, stream, dtype, nrm)
            assert rc == _lib.OK, msg
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for case, ref, pair in zip(CASES, refs, outs):
        for out in pair:
            got = out.cpu().numpy().reshape(case[0], order="F")
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err <= tol, (case[0], err)


def test_noalloc_rejects_oversized_and_host_output():
    torch = pytest.importorskip("torch")
    out = torch.empty(16, dtype=torch.float32, device="cuda")
    rc, msg = _noalloc(out, (300, 300, 300), (1024, 1024, 1024), (1, 1, 1), (9, 9, 9), 3, 0.5, 1, 0)
    assert rc == _lib.EINVAL and "64 MiB" in msg
    host = np.zeros(64, dtype=np.float32)
    msg = C.create_string_buffer(256)
    rc = _lib.lib().scarl_gen_padded_noalloc(C.c_void_p(host.ctypes.data), S.F32, _i3((4, 4, 4)),
                                             None, _d3((1, 1, 1)), _d3((1, 1, 1)), 1, 0.5, 1, 0, 0,
                                             None, msg, 256)
    assert rc == _lib.EINVAL and "device memory" in msg.value.decode()


def test_noalloc_rejects_other_gpu_output():
    """A device pointer of another GPU is rejected before any work is queued
    (needs two visible GPUs)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU visible")
    other = torch.empty(64, dtype=torch.float32, device="cuda:1")
    torch.cuda.set_device(0)
    rc, msg = _noalloc(other, (4, 4, 4), None, (1, 1, 1), (2, 2, 2), 1, 0.5, 1, 0)
    assert rc == _lib.EINVAL and "current GPU" in msg
