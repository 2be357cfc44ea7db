"""The native 64^3-512^3 real FFT (pm_rfft3_native / pm_irfft3_native) against torch's cuFFT
in float64, and the engine's native-transform step (Green multiply fused into the inverse)
against its cuFFT step on the same particles."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
N = 256


def _rel(a, b):
    return float((a - b).abs().pow(2).sum().sqrt() / b.abs().pow(2).sum().sqrt())


@pytest.mark.parametrize("n,nf", [(64, 3), (128, 2), (256, 2), (512, 1)])
def test_forward_and_inverse_match_cufft(n, nf):
    import torch
    from pbh_b200 import _lib
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((nf, n, n, n), device="cuda", generator=g, dtype=torch.float32)
    spec = torch.empty((nf, n // 2 + 1, n, n), dtype=torch.complex64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(lib.pm_rfft3_native(n, x.data_ptr(), spec.data_ptr(), nf, None), "pm_rfft3_native")
    torch.cuda.synchronize()
    for f in range(nf):                                                     # [kz][kx][ky]
        ref = torch.fft.rfftn(x[f].double()).permute(2, 0, 1)
        assert _rel(spec[f].to(torch.complex128), ref) < 2e-6
        del ref
    work = torch.empty_like(spec)
    back = torch.empty_like(x)
    _lib.check(lib.pm_irfft3_native(n, spec.data_ptr(), work.data_ptr(), back.data_ptr(), nf, None), "pm_irfft3_native")
    torch.cuda.synchronize()
    assert _rel(back.double() / n ** 3, x.double()) < 2e-6
    if n == N:
        # the n = 256 forms give the same bits
        spec2 = torch.empty_like(spec)
        _lib.check(lib.pm_rfft3_256(x.data_ptr(), spec2.data_ptr(), nf, None), "pm_rfft3_256")
        torch.cuda.synchronize()
        assert torch.equal(spec2, spec)
    # an arbitrary (not Hermitian-consistent) spectrum: the inverse equals irfftn's (which uses
    # the real parts of the kz = 0 and n/2 lines after the x-y inverse, like any C2R)
    s2 = torch.randn((1, n // 2 + 1, n, n), dtype=torch.complex64, device="cuda", generator=g)
    out = torch.empty((1, n, n, n), dtype=torch.float32, device="cuda")
    _lib.check(lib.pm_irfft3_native(n, s2.data_ptr(), work.data_ptr(), out.data_ptr(), 1, None), "pm_irfft3_native")
    torch.cuda.synchronize()
    full = s2[0].to(torch.complex128).permute(1, 2, 0)                      # [kx][ky][kz]
    t = torch.fft.ifft(torch.fft.ifft(full, dim=0), dim=1) * (n * n)        # x-y inverse, unnormalised
    t[..., 0] = t[..., 0].real.to(torch.complex128)
    t[..., n // 2] = t[..., n // 2].real.to(torch.complex128)
    ref2 = torch.fft.irfft(t, n=n, dim=2) * n
    assert _rel(out[0].double(), ref2) < 2e-6


def test_engine_native_transform_matches_cufft_step():
    import torch
    from pbh_b200 import recipe
    from pbh_b200.engine import Engine, PeakConfig
    from pbh_b200.ic import recipe_particles
    spec = recipe.single_peak(N=N, steps=20, seed=9)
    x, p = recipe_particles(spec, device=0, device_noise=True)
    res = []
    for native in (False, True):
        eng = Engine([PeakConfig(N=N, Np=N, L=1.0)], native_fft=native)
        eng.set_particles(0, x, p, 1.0, mode=0, param=spec.ratio(), max_steps=20)
        eng.run(1)                                   # prime: deposit and forces at the loaded positions
        r = dict(delta=eng.delta(0).double(), acc=eng.acc(0, 1.0).double())
        eng.run(3)                                   # three pushes with these forces and their successors
        r.update(pos=eng.particles(0)[0], st=eng.stats(0))
        res.append(r)
        eng.close()
    a, b = res
    assert torch.equal(a["delta"], b["delta"])       # same positions: the deposit does not involve the FFT
    assert _rel(b["acc"], a["acc"]) < 1e-5
    # after a few steps the two runs differ by the FP32 rounding of their forces only
    assert float((b["pos"] - a["pos"]).abs().max()) * N < 1e-5   # in cells
    assert b["st"].potential == pytest.approx(a["st"].potential, rel=1e-5)
    assert b["st"].status == 0


def test_native_transform_in_a_mixed_served_engine():
    """Served (dynamic) mode with meshes of two sizes and an idle 256^3 slot below an occupied
    one: the native transform's slot mapping and Green partials against cuFFT's."""
    import torch
    from pbh_b200 import recipe
    from pbh_b200.engine import Engine, PeakConfig
    from pbh_b200.ic import recipe_particles
    cfgs = [PeakConfig(N=32, Np=32, L=1.0), PeakConfig(N=N, Np=N, L=1.0), PeakConfig(N=N, Np=N, L=1.0)]
    loads = {0: recipe.single_peak(N=32, steps=20, seed=5), 2: recipe.single_peak(N=N, steps=20, seed=6)}
    res = []
    for native in (False, True):
        eng = Engine(cfgs, graph=False, dynamic=True, native_fft=native)
        for i, spec in loads.items():
            x, p = recipe_particles(spec, device=0, device_noise=True)
            eng.set_particles(i, x, p, 1.0, mode=0, param=spec.ratio(), max_steps=20)
            del x, p
        eng.run(1)
        res.append({i: (eng.acc(i, 1.0).double(), eng.stats(i)) for i in loads})
        eng.close()
    for i in loads:
        (a_cu, s_cu), (a_na, s_na) = res[0][i], res[1][i]
        assert _rel(a_na, a_cu) < 1e-5
        assert s_na.potential == pytest.approx(s_cu.potential, rel=1e-5)
        assert s_na.status == 0
