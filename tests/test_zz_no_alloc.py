"""GPU test of vis_fourier_slice_sum_noalloc, the entry point for callers that
cannot allocate device memory (fixed device footprint, per-frame render loops,
memory owned by another framework's pool).  It keeps its scratch in a fixed
array of the library's device image and must give what the allocating path
gives.

The test calls it through the C ABI on caller-owned device buffers, twice in a
row (the second call meets the first call's leftovers in the shared scratch),
then a third time adding into the output (accumulate != 0), for three kernel
variants: a Wendland group with radii (Phi^ table), an SPH group without radii
(Phi^ applied per sample) and a decaying Gaussian with radii.
Each result, taken through an unnormalised 2D C2R, is compared with the image
that vis_fourier_volume_rendering renders for the same group and view (the
slice itself cannot be read back from that path: cuFFT's C2R may overwrite
its input), and the slice is compared with the FP64 oracle, within the
tolerance the other parity tests use.

The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from libmeshlessvis_b200 import _lib as L
from libmeshlessvis_b200 import meshless as M
from libmeshlessvis_b200.workloads import constraints

from util import to_dataset

pytestmark = pytest.mark.gpu

SPEC_TOL = 1e-5


# (basis, per-particle radii?): the cubic Phi^-table kernel with radii, the
# factored kernel without radii (Phi^ applied per sample in the finalize), and
# the exp2 amplitude kernel of the decaying Gaussian
CASES = [(M.WENDLAND_D3_C2, True), (M.SPH, False), (M.GAUSSIAN_DECAYING, True)]


@pytest.mark.parametrize("basis,with_radii", CASES)
def test_noalloc_slice_matches_allocating_path_on_two_calls(basis, with_radii):
    import torch

    lib = M.lib()
    rng = np.random.default_rng(31)
    n = 5003
    cons = constraints(rng.random((n, 3), dtype=np.float32), rng.standard_normal(n).astype(np.float32))
    radii = np.exp(rng.uniform(np.log(0.01), np.log(0.05), n)).astype(np.float32) if with_radii else None
    step, cutoff, samples = ((1.0, 1.0), (24, 16), (64, 40)) if with_radii else ((0.05, 0.05), (24, 16), (64, 40))
    u, v = (0.8, 0.0, -0.6), (0.0, 1.0, 0.0)
    nx, ny = samples

    # the existing, allocating entry point
    cfg = M.Config(step=step, cutoff=cutoff, u=u, v=v, samples=samples, block_length=64)
    ds = to_dataset([(cons, radii, basis)])
    cfg.register(ds)
    cfg.render(ds)
    ref_image = cfg.image()
    cfg.unregister(ds)
    cfg.close()
    ref_slice = O.arrange(O.slice_sum(cons, radii, basis, step, cutoff, u, v), cutoff, samples)

    # caller-owned device inputs and output
    d_cons = torch.from_numpy(cons.view(np.float32).reshape(n, 4).copy()).cuda()
    d_radii = torch.from_numpy(radii).cuda() if with_radii else None
    d_out = torch.zeros((nx, ny // 2 + 1, 2), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call(accumulate):
        rc = lib.vis_fourier_slice_sum_noalloc(d_cons.data_ptr(), None if d_radii is None else d_radii.data_ptr(), n,
                                               basis, L.float2(*step), L.int2(*cutoff), L.float3(*u), L.float3(*v),
                                               L.int2(*samples), d_out.data_ptr(), accumulate, stream)
        assert rc == 0, lib.vis_get_last_error_message()
        torch.cuda.synchronize()
        return d_out.cpu().numpy().view(np.complex64)[..., 0].copy()

    results = []
    for _ in range(2):
        got = call(0)
        image = torch.fft.irfft2(torch.view_as_complex(d_out), s=(nx, ny), norm="forward").cpu().numpy()
        assert O.rel_l2(image, ref_image) < SPEC_TOL
        assert O.rel_l2(got, ref_slice) < SPEC_TOL
        results.append(got)
    np.testing.assert_array_equal(results[0], results[1])
    # accumulate != 0 adds the slice to what the buffer holds: twice the slice
    twice = call(1)
    assert O.rel_l2(twice, 2.0 * ref_slice) < SPEC_TOL
    np.testing.assert_allclose(twice, 2.0 * results[0], rtol=1e-6, atol=1e-6 * np.abs(results[0]).max())


def test_noalloc_rejects_bad_arguments_without_launching():
    lib = M.lib()
    before = lib.vis_kernel_launch_count()
    rc = lib.vis_fourier_slice_sum_noalloc(None, None, 10, M.SPH, L.float2(1, 1), L.int2(8, 8), L.float3(1, 0, 0),
                                           L.float3(0, 1, 0), L.int2(16, 16), None, 0, None)
    assert rc == 1
    # a slice larger than the fixed scratch is refused with a clear error
    big = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.vis_fourier_slice_sum_noalloc(big, None, 1, M.SPH, L.float2(1, 1), L.int2(2048, 2048),
                                           L.float3(1, 0, 0), L.float3(0, 1, 0), L.int2(4096, 4096), big, 0, None)
    assert rc == 1
    assert b"no-alloc scratch" in lib.vis_get_last_error_message()
    lib.vis_clear_last_error()
    assert lib.vis_kernel_launch_count() == before
