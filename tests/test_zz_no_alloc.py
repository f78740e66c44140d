"""lenia_fft_step_noalloc: one spectral substep on caller-owned device buffers
with all scratch in the library's fixed static device array.

This entry point exists for callers that cannot allocate device memory where
they step the field (a real-time frame callback, where an allocation could
synchronise the device and stall the frame, or a host that reserves the GPU's
memory up front). These tests call it through the C ABI and compare it with
the regular context-owning entry point (lenia_step) on the same inputs, for
two calls in a row, at one size that uses the compile-time-plan kernels
(128x64), one that uses the runtime-plan kernels (120x90) and with the
implicit kernel of a config without a kernels list; and check that repeated
calls leave the device's free memory unchanged. The file is named to be
collected last; it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

import life_simulation_b200 as lb

pytestmark = pytest.mark.gpu

TOL = 1e-6  # same inputs, same kernels: differences are at most rounding


def _pcg(v: int) -> int:
    state = (v * 747796405 + 2891336453) & 0xFFFFFFFF
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & 0xFFFFFFFF
    return (word >> 22) ^ word


def _substep_seed(reset_seed: int, frame: int) -> int:
    # deriveSeed(seed, "LEN1") then pcgHash(seed_ ^ (frame*197 + 0)).
    s = _pcg(reset_seed ^ _pcg(0x4C454E31))
    return _pcg(s ^ ((frame * 197) & 0xFFFFFFFF))


PARAMS = {
    "convMode": "fft", "fftAnySize": True, "radius": 9, "dt": 0.2, "growthMode": 0,
    "noiseAmount": 0.3, "muJitter": 0.5, "injectAmount": 0.0,
    "kernels": [{"radiusScale": 1.0, "mu": 0.15, "sigma": 0.02, "weight": 0.6, "betas": [1.0]},
                {"radiusScale": 0.6, "mu": 0.25, "sigma": 0.04, "weight": 0.4, "betas": [1.0, 0.5]}],
}


# Without a "kernels" list: one implicit kernel from the frame's growth mu
# and sigma (num_kernels == 0 in the C config).
PARAMS_IMPLICIT = {
    "convMode": "fft", "fftAnySize": True, "radius": 9, "dt": 0.2, "growthMode": 1,
    "growthMu": 0.2, "growthSigma": 0.03, "noiseAmount": 0.0, "muJitter": 0.0, "injectAmount": 0.0,
}


@pytest.mark.parametrize("w,h,params", [(128, 64, PARAMS), (120, 90, PARAMS), (128, 64, PARAMS_IMPLICIT)],
                         ids=["fast-plan", "runtime-plan", "implicit-kernel"])
def test_noalloc_matches_context_entry_point_two_calls(w, h, params):
    import torch

    L = lb.load_library()
    p = dict(params, simWidth=w, simHeight=h)
    init = np.random.default_rng(w + h).random((h, w)).astype(np.float32) * 0.6

    ref = lb.LeniaModule(p, w, h)
    ref.reset(11)
    ref.upload(init)
    cfg = lb.config_from_params(p)

    dev = torch.device("cuda:0")
    a = torch.from_numpy(init).to(dev)
    b = torch.empty_like(a)
    stream = torch.cuda.current_stream().cuda_stream
    for frame in range(2):
        fp = ref.frame_params(frame)
        ref.step(fp, 1)
        want = ref.field()
        rc = L.lenia_fft_step_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), w, h,
                                      ctypes.byref(cfg), ctypes.byref(fp), _substep_seed(11, frame),
                                      ctypes.c_void_p(stream) if stream else None)
        assert rc == 0, L.lenia_noalloc_last_message().decode()
        torch.cuda.synchronize()
        got = b.cpu().numpy()
        assert np.abs(got - want).max() <= TOL, (w, h, frame, float(np.abs(got - want).max()))
        a, b = b, a
    ref.close()


def test_noalloc_allocates_no_device_memory():
    """The defining property: once the library's module (and its static
    array) is resident after a first call, further calls leave the device's
    free memory unchanged."""
    import torch

    L = lb.load_library()
    w, h = 128, 64
    p = dict(PARAMS, simWidth=w, simHeight=h)
    cfg = lb.config_from_params(p)
    fp = lb.make_frame_params(dt=0.2, growth_sigma=0.02)
    a = torch.rand((h, w), device="cuda:0")
    b = torch.empty_like(a)

    def call(src, dst):
        rc = L.lenia_fft_step_noalloc(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), w, h,
                                      ctypes.byref(cfg), ctypes.byref(fp), 5, None)
        assert rc == 0, L.lenia_noalloc_last_message().decode()

    call(a, b)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(4):
        call(a, b)
        call(b, a)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_rejects_fields_beyond_the_scratch():
    import torch

    L = lb.load_library()
    w, h = 1920, 1080
    p = dict(PARAMS, simWidth=w, simHeight=h)
    cfg = lb.config_from_params(p)
    fp = lb.make_frame_params(growth_sigma=0.02)
    a = torch.zeros((h, w), device="cuda:0")
    b = torch.empty_like(a)
    rc = L.lenia_fft_step_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), w, h,
                                  ctypes.byref(cfg), ctypes.byref(fp), 1, None)
    assert rc == -2  # LENIA_ERR_UNSUPPORTED
    assert b"too large" in L.lenia_noalloc_last_message()
