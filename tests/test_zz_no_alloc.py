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


def _noalloc(out, Np, pad, dx, cl, cm, nu, seed, stream, dtype=S.F32):
    msg = C.create_string_buffer(256)
    rc = _lib.lib().scarl_gen_padded_noalloc(C.c_void_p(out.data_ptr()), dtype, _i3(Np),
                                             _i3(pad) if pad else None, _d3(dx), _d3(cl), cm, nu,
                                             1, seed, stream, None, msg, 256)
    return rc, msg.value.decode()


CASES = [  # Np, pad, xStep, corrL, corrMod, nu, seed, stream
    ((60, 50, 40), (128, 128, 128), (1.0, 1.0, 1.0), (8.0, 6.0, 5.0), 3, 0.5, 11, 0),
    ((100, 33, 70), (256, 64, 128), (0.5, 1.0, 1.0), (9.0, 4.0, 7.0), 1, 0.5, 12345, 3),
]


@pytest.mark.parametrize("dtype,tol", [(S.F32, 1e-6), (S.F64, 1e-13)])
def test_noalloc_matches_allocating_entry_point_twice(ctx, dtype, tol):
    torch = pytest.importorskip("torch")
    tdt = torch.float32 if dtype == S.F32 else torch.float64
    for Np, pad, dx, cl, cm, nu, seed, stream in CASES:
        ref = S.gen_padded(ctx, Np, dx, cl, cm, nu, pad=pad, seed=seed, stream=stream, dtype=dtype)
        out = torch.full((int(np.prod(Np)),), float("nan"), dtype=tdt, device="cuda")
        rc, msg = _noalloc(out, Np, pad, dx, cl, cm, nu, seed, stream, dtype)
        assert rc == _lib.OK, msg
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(Np, order="F")
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= tol, (Np, err)


def test_noalloc_rejects_oversized_and_host_output():
    torch = pytest.importorskip("torch")
    out = torch.empty(16, dtype=torch.float32, device="cuda")
    rc, msg = _noalloc(out, (300, 300, 300), (1024, 1024, 1024), (1, 1, 1), (9, 9, 9), 3, 0.5, 1, 0)
    assert rc == _lib.EINVAL and "64 MiB" in msg
    host = np.zeros(8, dtype=np.float32)
    msg = C.create_string_buffer(256)
    rc = _lib.lib().scarl_gen_padded_noalloc(C.c_void_p(host.ctypes.data), S.F32, _i3((2, 2, 2)),
                                             None, _d3((1, 1, 1)), _d3((1, 1, 1)), 1, 0.5, 1, 0, 0,
                                             None, msg, 256)
    assert rc == _lib.EINVAL and "device memory" in msg.value.decode()
