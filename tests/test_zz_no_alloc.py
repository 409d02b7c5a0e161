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


def _call(L, d_in, d_out, nr, nt, dt, band, err):
    b = [C.c_float(v) for v in band]
    rc = L.daw_filmartin2d_noalloc(C.c_void_p(d_in), nr, nt, dt, *[C.byref(v) for v in b],
                                   C.c_void_p(d_out), None, err, len(err))
    return rc, tuple(v.value for v in b)


def test_noalloc_filter_matches_regular_entry_point_twice(pkg):
    torch = pytest.importorskip("torch")
    L = pkg.lib()
    err = C.create_string_buffer(512)
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
            rc, band = _call(L, d_in.data_ptr(), d_out.data_ptr(), nr, nt, dt, c["band"], err)
            assert rc == 0, err.value.decode()
            y = d_out.cpu().numpy().T
            assert np.isfinite(y).all()
            assert rel_l2(y, ref) <= TOL, (nt, rel_l2(y, ref))
            assert band == ref_band


def test_noalloc_filter_rejects_traces_beyond_its_work_space(pkg):
    torch = pytest.importorskip("torch")
    L = pkg.lib()
    err = C.create_string_buffer(512)
    d = torch.zeros(16, device="cuda:0")
    # 70000 samples need nto = 131072: more weights than the fixed array holds
    rc, _ = _call(L, d.data_ptr(), d.data_ptr(), 1, 70000, 4e-4, (5.0, 30.0, 5.0, 5.0), err)
    assert rc == -1  # DAW_ERR_ARG
    assert b"exceeds the maximum of 65536 samples" in err.value
