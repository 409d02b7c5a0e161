"""daw_filmartin2d_noalloc, the filter entry point that allocates no GPU
memory, against the regular daw_filmartin2d, through the C ABI.

The no-allocation variant is for callers that cannot call cudaMalloc when
they filter: a shot batch of this library or a framework's caching allocator
already holds the HBM, or the caller must not stall its other streams with
the device-wide synchronisation of cudaMalloc/cudaFree.  They pass their own
device buffers, and the work space is a fixed array inside the library that
every call shares.  Two calls in a row, with different trace lengths, check
that what the first call leaves in that array does not change the second
one's result.

The file name sorts last, so a run that stops at its first failure has run
every other test before this one.  It runs alone as well:
    python -m pytest tests/test_zz_no_alloc.py -m gpu
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6  # the filter tests' bar (rel. L2)

CASES = [
    # 7500 samples: nto 8192, the transform stays in shared memory; the
    # fixed array holds the weights only
    dict(nt=7500, nr=37, dt=4e-4, band=(7.5, 37.5, 7.5, 7.5), seed=11),
    # 20000 samples: nto 32768, FFT work space in the fixed array, 29 traces
    # in several launches; fhig above Nyquist exercises the in-place clamp
    dict(nt=20000, nr=29, dt=2e-3, band=(5.0, 300.0, 2.0, 5.0), seed=12),
]


def _call(L, d_in, d_out, nr, nt, dt, band, err, stream=None):
    b = [C.c_float(v) for v in band]
    rc = L.daw_filmartin2d_noalloc(C.c_void_p(d_in), nr, nt, dt, *[C.byref(v) for v in b],
                                   C.c_void_p(d_out), C.c_void_p(stream), err, len(err))
    return rc, tuple(v.value for v in b)


@pytest.mark.parametrize("on_stream", [False, True])
def test_noalloc_filter_matches_regular_entry_point_twice(pkg, on_stream):
    """Both cases in a row; on the legacy default stream, and on a stream of
    the caller's (a torch stream), which the call must honour: the output is
    read back on that stream after the call returns."""
    torch = pytest.importorskip("torch")
    L = pkg.lib()
    err = C.create_string_buffer(512)
    stream = torch.cuda.Stream(device=0) if on_stream else None
    with pkg.Handle(0, preset="mixed") as h:
        for c in CASES:
            nt, nr, dt = c["nt"], c["nr"], c["dt"]
            x = np.asfortranarray(
                np.random.default_rng(c["seed"]).standard_normal((nt, nr)).astype(np.float32))
            ref, ref_band = h.filmartin2d(x, dt, *c["band"])
            # (nt, nr) column-major == (nr, nt) row-major
            d_in = torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda:0")
            d_out = torch.full_like(d_in, float("nan"))
            torch.cuda.synchronize()
            rc, band = _call(L, d_in.data_ptr(), d_out.data_ptr(), nr, nt, dt, c["band"], err,
                             stream.cuda_stream if stream is not None else None)
            assert rc == 0, err.value.decode()
            if stream is not None:
                with torch.cuda.stream(stream):
                    y = d_out.cpu().numpy().T
            else:
                y = d_out.cpu().numpy().T
            assert np.isfinite(y).all()
            assert rel_l2(y, ref) <= TOL, (nt, rel_l2(y, ref))
            assert band == ref_band


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, {root!r})
import __graft_entry__ as e
pkg = e.load_package()
L = pkg.lib()
nt, nr = 20000, 5
x = torch.randn(nr, nt, device="cuda:0")
y = torch.empty_like(x)
torch.cuda.synchronize()
b = [C.c_float(v) for v in (5.0, 30.0, 5.0, 5.0)]
err = C.create_string_buffer(256)
def call(nr_, xin, yout):
    return L.daw_filmartin2d_noalloc(C.c_void_p(xin), nr_, nt, 2e-3,
                                     *[C.byref(v) for v in b], C.c_void_p(yout), None, err, 256)
if {with_handle}:
    h = C.c_void_p()
    assert L.daw_create(C.byref(h), 0) == 0
else:
    assert call(0, None, None) == 0, err.value   # the documented set-up call
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info(0)[0]
rc = call(nr, x.data_ptr(), y.data_ptr())
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info(0)[0]
assert rc == 0, err.value
assert torch.isfinite(y).all()
print("free before", free0, "after", free1)
assert free1 == free0, (free0, free1)
"""


@pytest.mark.parametrize("with_handle", [True, False])
def test_noalloc_first_call_allocates_nothing(with_handle):
    """In a fresh process, after daw_create on the device (or after the
    documented set-up call with nr = 0 when no handle exists), the first
    filtering call leaves the device's free memory unchanged: the fixed work
    space and the filter kernel's code were placed before it.  Traces of
    20000 samples use the FFT work space inside the fixed array."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH.format(root=root, with_handle=with_handle)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_noalloc_filter_rejects_traces_beyond_its_work_space(pkg):
    torch = pytest.importorskip("torch")
    L = pkg.lib()
    err = C.create_string_buffer(512)
    d = torch.zeros(16, device="cuda:0")
    # 70000 samples need nto = 131072: more weights than the fixed array holds
    rc, _ = _call(L, d.data_ptr(), d.data_ptr(), 1, 70000, 4e-4, (5.0, 30.0, 5.0, 5.0), err)
    assert rc == -1  # DAW_ERR_ARG
    assert b"exceeds the maximum of 65536 samples" in err.value
