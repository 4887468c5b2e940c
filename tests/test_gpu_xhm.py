"""IMRPhenomXHM on the kernels against the golden vectors of the reference's
own code (``tests/golden/xhm_*.npz``, made by ``make_golden_xhm.py``):
the set-up's tables (the higher modes in the layout of the reference's
MODE_LAYOUT, ``models/xhm/core.py:78-113``), the five modes and the
polarizations (``models/xhm/core.py:524-556``).

Bars: FP64 tables 1e-9 relative to each field's scale; FP64 modes and
polarizations 1e-9 relative to each series' peak (the reference's float64
evaluation); FP32 polarizations a mismatch below 1e-6 and a phase error
below 1e-3 rad where the amplitude is above 1e-3 of its peak for mass
ratios below 50 (the path's FP32 bar), 1e-2 rad beyond: the inspiral
terms after the leading one, carried in float, scale as 1 / eta (10^3 to
10^4 rad at a mass ratio of 100, whose float rounding alone is ~1e-3 rad;
the (2,2) of IMRPhenomXAS's FP32 form shows the same).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import compare, golden

pytestmark = pytest.mark.gpu

# (name, length) of the fields of a mode's table (models/xhm/core.py:98-113)
FIELDS = [("phase", 54), ("sph", 4), ("atan_a", 3), ("atan_w", 3), ("shift", 1), ("f_phase_in", 1),
          ("f_phase_im", 1), ("f_amp_in", 1), ("f_amp_im", 1), ("pn_re", 7), ("pn_im", 7), ("pseudo", 3),
          ("inter", 8), ("inter_c", 1), ("inter_h", 1), ("rd", 3), ("falloff", 3), ("aux", 4), ("f_aux", 1),
          ("mix", 4), ("on", 1)]
REF_HEAD = 86  # the reference's table: its XAS table (86), then factors, amp0, s, the modes


def _run(cuda, params, grid, *, precision, amp_scale=1e21, reference_mf=None, t_c=None):
    import torch

    from waveformx_b200 import _lib, ops

    real = torch.float32 if precision == _lib.FP32 else torch.float64
    p = torch.as_tensor(np.atleast_2d(params), dtype=torch.float64, device=cuda)
    f = torch.as_tensor(np.asarray(grid), dtype=real, device=cuda)
    tables = ops.setup("IMRPhenomXHM", p, f[:1].double(), amp_scale=amp_scale, reference_mf=reference_mf,
                       precision=precision)
    tc = None if t_c is None else torch.as_tensor(np.atleast_1d(t_c), dtype=real, device=cuda)
    hp, hc, modes = ops.xhm_modes(tables.table, f, tc)
    return tables, hp.cpu().numpy(), hc.cpu().numpy(), modes.cpu().numpy()


def _each(data):
    """(params, grid) of each binary of a fixture."""
    f = data["frequencies"]
    for b, p in enumerate(data["params"]):
        yield b, p, (f[b] if f.ndim == 2 else f)


def _options(name):
    return {"reference_mf": dict(reference_mf=0.01), "unscaled": dict(amp_scale=1.0)}.get(name, {})


def _peak_relative(a, b):
    scale = np.max(np.abs(b))
    return np.max(np.abs(a - b)) / scale if scale > 0 else np.max(np.abs(a))


@pytest.mark.parametrize("name", ["cases", "random", "reference_mf", "unscaled"])
def test_tables_match_the_reference(cuda, name):
    from waveformx_b200 import _lib

    data = golden(f"xhm_{name}")
    for b, p, grid in _each(data):
        tables, *_ = _run(cuda, p, grid, precision=_lib.FP64, **_options(name))
        got = tables.table.cpu().numpy()[0]
        ref = data["tables"][b]
        np.testing.assert_allclose(got[72:92], ref[REF_HEAD:REF_HEAD + 20], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(got[92:94], ref[REF_HEAD + 20:REF_HEAD + 22], rtol=1e-14)
        for m in range(4):
            mine = got[96 + 112 * m: 96 + 112 * (m + 1)]
            theirs = ref[REF_HEAD + 22 + 112 * m: REF_HEAD + 22 + 112 * (m + 1)]
            at = 0
            for field, n in FIELDS:
                a, r = mine[at:at + n], theirs[at:at + n]
                scale = max(np.max(np.abs(r)), 1e-300)
                assert np.max(np.abs(a - r)) <= 1e-9 * scale, (name, b, m, field, a, r)
                at += n
        assert int(tables.status.cpu()[0]) == 0


@pytest.mark.parametrize("name", ["cases", "random", "reference_mf", "unscaled"])
def test_fp64_modes_and_polarizations(cuda, name):
    from waveformx_b200 import _lib

    data = golden(f"xhm_{name}")
    for b, p, grid in _each(data):
        _, hp, hc, modes = _run(cuda, p, grid, precision=_lib.FP64, **_options(name))
        for k in range(5):
            err = _peak_relative(modes[0, k], data["modes"][b, k])
            assert err < 1e-9, (name, b, k, err)
        assert _peak_relative(hp[0], data["hplus"][b]) < 1e-9
        assert _peak_relative(hc[0], data["hcross"][b]) < 1e-9


@pytest.mark.parametrize("name", ["cases", "random"])
def test_fp32_polarizations(cuda, name):
    from waveformx_b200 import _lib

    data = golden(f"xhm_{name}")
    for b, p, grid in _each(data):
        _, hp, hc, _ = _run(cuda, p, grid, precision=_lib.FP32)
        for got, ref in ((hp[0], data["hplus"][b]), (hc[0], data["hcross"][b])):
            _, mismatch = compare(got.astype(np.complex128), ref)
            assert mismatch < 1e-6, (name, b, mismatch)
            big = np.abs(ref) > 1e-3 * np.max(np.abs(ref))
            dphi = np.angle(got[big] * np.conj(ref[big]))
            q = max(p[0], p[1]) / min(p[0], p[1])
            assert np.max(np.abs(dphi)) < (1e-3 if q < 50 else 1e-2), (name, b, q, np.max(np.abs(dphi)))


def test_t_c_is_a_phase(cuda):
    """t_c multiplies every mode by exp(-2 pi i f t_c)."""
    from waveformx_b200 import _lib

    data = golden("xhm_random")
    p, grid = data["params"][:3], data["frequencies"]
    tc = np.array([0.0, 0.05, -0.0931])
    for precision, tol in ((_lib.FP64, 1e-12), (_lib.FP32, 2e-5)):
        _, hp0, _, m0 = _run(cuda, p, grid, precision=precision)
        _, hp1, _, m1 = _run(cuda, p, grid, precision=precision, t_c=tc)
        shift = np.exp(-2j * np.pi * grid[None, :] * tc[:, None])
        assert _peak_relative(hp1, hp0 * shift) < tol
        assert _peak_relative(m1, m0 * shift[:, None, :]) < tol


def test_odd_modes_vanish_for_equal_binaries(cuda):
    """Equal masses and spins: (2,1) and (3,3) are zero (models/xhm/core.py:383-389)."""
    from waveformx_b200 import _lib

    grid = np.geomspace(20.0, 700.0, 200)
    for precision in (_lib.FP64, _lib.FP32):
        _, _, _, modes = _run(cuda, [30.0, 30.0, 0.2, 0.2, 400.0, 0.4, 0.0, 20.0], grid, precision=precision)
        assert np.all(modes[0, 1] == 0) and np.all(modes[0, 2] == 0)
        assert np.max(np.abs(modes[0, 3])) > 0 and np.max(np.abs(modes[0, 4])) > 0


def test_batch_equals_single(cuda):
    """A batch on one grid: each row its binary alone (FP64, bit for bit)."""
    from waveformx_b200 import _lib

    data = golden("xhm_random")
    _, hp, hc, modes = _run(cuda, data["params"], data["frequencies"], precision=_lib.FP64)
    for b in (0, 7, 23):
        _, hp1, hc1, m1 = _run(cuda, data["params"][b], data["frequencies"], precision=_lib.FP64)
        np.testing.assert_array_equal(hp[b], hp1[0])
        np.testing.assert_array_equal(modes[b], m1[0])


def test_drop_in_forward(cuda):
    """polarizations_function("IMRPhenomXHM"): the reference's call (its
    ``torch.py:175-183``) on the kernels, values and gradients."""
    import torch

    import waveformx_b200 as wb
    from waveformx_b200.torch import polarizations_function

    data = golden("xhm_random")
    p = data["params"][:4]
    grid = data["frequencies"]
    f = polarizations_function("IMRPhenomXHM")
    binary = dict(mass_1=torch.tensor(p[:, 0]), mass_2=torch.tensor(p[:, 1]),
                  spin_1=torch.tensor(np.stack([0 * p[:, 2], 0 * p[:, 2], p[:, 2]], -1)),
                  spin_2=torch.tensor(np.stack([0 * p[:, 3], 0 * p[:, 3], p[:, 3]], -1)),
                  luminosity_distance=torch.tensor(p[:, 4]), inclination=torch.tensor(p[:, 5]),
                  phi_ref=torch.tensor(p[:, 6]), f_ref=torch.tensor(p[:, 7]))
    hp, hc = f(binary, torch.tensor(grid, device=cuda))
    assert hp.dtype == torch.complex128 and hp.shape == (4, len(grid))
    assert _peak_relative(hp.cpu().numpy(), data["hplus"][:4]) < 1e-9
    assert _peak_relative(hc.cpu().numpy(), data["hcross"][:4]) < 1e-9
    # gradients: autograd through the backward kernel equals ops.xhm_vjp
    from waveformx_b200 import ops

    m1 = torch.tensor(p[:, 0], requires_grad=True)
    chi = torch.tensor(np.stack([0 * p[:, 2], 0 * p[:, 2], p[:, 2]], -1), requires_grad=True)
    hp, hc = f(dict(binary, mass_1=m1, spin_1=chi), torch.tensor(grid, device=cuda))
    rng = np.random.default_rng(9)
    a = torch.as_tensor(rng.normal(size=hp.shape) + 1j * rng.normal(size=hp.shape), device=hp.device)
    loss = (torch.conj(a) * hp).real.sum() + 2.0 * (torch.conj(a) * hc).real.sum()
    loss.backward()
    params = torch.as_tensor(p, device=cuda).contiguous()
    f64 = torch.as_tensor(grid, device=cuda)
    grad = ops.xhm_vjp(params, f64[:1], f64, None, None, a, 2.0 * a).cpu().numpy()
    np.testing.assert_allclose(m1.grad.cpu().numpy(), grad[:, 0], rtol=1e-12)
    np.testing.assert_allclose(chi.grad.cpu().numpy()[:, 2], grad[:, 2], rtol=1e-12)
    assert np.all(chi.grad.cpu().numpy()[:, :2] == 0)


def test_batch_polarizations(cuda):
    """batch_polarizations("IMRPhenomXHM", ...): the reference's batch call
    (its ``_api.py:307-360``) on a shared grid, FP64, and ragged (each binary
    on its own grid: the rows of the cases)."""
    import waveformx_b200 as wb

    data = golden("xhm_random")
    p = data["params"]
    columns = dict(mass_1=p[:, 0], mass_2=p[:, 1], spin_1x=0 * p[:, 0], spin_1y=0 * p[:, 0], spin_1z=p[:, 2],
                   spin_2x=0 * p[:, 0], spin_2y=0 * p[:, 0], spin_2z=p[:, 3], luminosity_distance=p[:, 4],
                   inclination=p[:, 5], phi_ref=p[:, 6], f_ref=p[:, 7])
    res = wb.batch_polarizations("IMRPhenomXHM", data["frequencies"], columns, output="numpy")
    assert res.ok.all()
    assert _peak_relative(np.asarray(res.hplus), data["hplus"]) < 1e-9
    assert _peak_relative(np.asarray(res.hcross), data["hcross"]) < 1e-9
    cases = golden("xhm_cases")
    q = cases["params"]
    grids = [cases["frequencies"][b][: 100 + 13 * b] for b in range(len(q))]
    columns = dict(mass_1=q[:, 0], mass_2=q[:, 1], spin_1x=0 * q[:, 0], spin_1y=0 * q[:, 0], spin_1z=q[:, 2],
                   spin_2x=0 * q[:, 0], spin_2y=0 * q[:, 0], spin_2z=q[:, 3], luminosity_distance=q[:, 4],
                   inclination=q[:, 5], phi_ref=q[:, 6], f_ref=q[:, 7])
    res = wb.batch_polarizations("IMRPhenomXHM", grids, columns, output="numpy")
    assert res.ok.all()
    for b, g in enumerate(grids):
        assert _peak_relative(np.asarray(res.hplus[b]), cases["hplus"][b][:len(g)]) < 1e-9
        assert _peak_relative(np.asarray(res.hcross[b]), cases["hcross"][b][:len(g)]) < 1e-9


# Binaries for the set-up's derivative: three of the golden draws, f_ref = 0
# (the first frequency stands for it), mass ratios either side of 20 (the
# inspiral amplitude's matching frequency switches to a blend with the
# extreme-mass-ratio cut at q >= 20, models/xhm/reference.py:118-140) and one
# on q = 20 exactly, where the derivative is the q >= 20 branch's.
JVP_BINARIES = np.array([
    [36.0, 29.0, 0.3, -0.1, 500.0, 0.7, 1.2, 20.0],
    [20.0, 15.5, 0.6, 0.2, 800.0, 0.3, 2.2, 0.0],
    [40.3, 2.0, 0.2, -0.7, 200.0, 2.9, 5.5, 30.0],
    [100.0, 5.2, 0.9, -0.9, 400.0, 1.3, 0.1, 20.0],
    [40.0, 2.0, -0.8, 0.4, 400.0, 1.3, 0.1, 0.0],
])


def _jvp_binaries():
    return np.concatenate([golden("xhm_random")["params"][:3], JVP_BINARIES])


def test_setup_jvp_against_differences(cuda):
    """The set-up on dual numbers (wfx_xhm_setup_jvp: d row64 / d params of
    every slot, the (2,2) table, the head, the four higher modes) against
    fourth-order central differences of the FP64 set-up, steps of 1e-4 of
    each value; on q = 20 second-order one-sided differences toward larger q
    along the masses, steps of 1e-6. Bar per slot: 1e-6 of the difference, plus 1e-9 of
    the largest tangent of the slot's part (head, (2,2), mode) and the
    difference's rounding (1e4 ulp of the value over the step). Along f_ref
    = 0 the column is zero."""
    import torch

    from waveformx_b200 import _lib, ops

    p = _jvp_binaries()
    batch = len(p)
    dev = cuda
    f_min = torch.tensor([20.0], dtype=torch.float64, device=dev)

    def rows(q):
        t = ops.setup("IMRPhenomXHM", torch.as_tensor(q, device=dev), f_min, precision=_lib.FP64)
        assert int(t.status.abs().sum()) == 0
        return t.table.cpu().numpy()

    tables = ops.setup("IMRPhenomXHM", torch.as_tensor(p, device=dev), f_min, precision=_lib.FP64, jvp=True)
    dtable = tables.dtable.cpu().numpy()
    assert dtable.shape == (batch, _lib.XHM_STRIDE64, 8)
    np.testing.assert_array_equal(tables.table.cpu().numpy(), rows(p))
    np.testing.assert_array_equal(ops.xhm_dtable(torch.as_tensor(p, device=dev), f_min).cpu().numpy(), dtable)
    base = rows(p)
    on_branch = p[:, 0] == 20.0 * p[:, 1]
    assert on_branch.sum() == 1 and (p[:, 0] / p[:, 1] > 20.0).sum() == 1
    parts = np.concatenate([np.zeros(72, int), np.ones(24, int), 2 + np.arange(4 * 112) // 112])
    for j in range(8):
        h = 1e-4 * np.maximum(1.0, np.abs(p[:, j]))

        def at(k, step):
            q = p.copy()
            q[:, j] += k * step
            return rows(q)

        fd = (8.0 * (at(1, h) - at(-1, h)) - (at(2, h) - at(-2, h))) / (12.0 * h[:, None])
        if j < 2:
            # (steps of 1e-6: the one-sided difference's truncation, (step
            # dA/dm)^2 for the cos and sin of the anchor A, is 1e-3 at 1e-4)
            side = 1.0 if j == 0 else -1.0
            hs = side * 1e-6 * np.maximum(1.0, np.abs(p[:, j]))
            one = (-3.0 * base + 4.0 * at(1, hs) - at(2, hs)) / (2.0 * hs[:, None])
            fd[on_branch] = one[on_branch]
            h = np.where(on_branch, np.abs(hs), h)
        tangent = dtable[:, :, j]
        if j == 7:
            zero = p[:, 7] == 0.0
            assert np.all(tangent[zero] == 0.0)
            fd[zero] = 0.0
        scale = np.stack([np.abs(tangent[:, parts == g]).max(axis=1) for g in range(6)], axis=1)[:, parts]
        bar = 1e-6 * np.abs(fd) + 1e-9 * scale + 1e4 * 2.2e-16 * np.abs(base) / h[:, None]
        bad = np.argwhere(~(np.abs(tangent - fd) <= bar))
        assert bad.size == 0, [(j, b, k, tangent[b, k], fd[b, k]) for b, k in bad[:5]]


def test_setup_jvp_on_random_draws(cuda):
    """The set-up on dual numbers against differences of the FP64 set-up for
    128 binaries drawn as the batch draws them: every slot and parameter
    matches fourth-order central differences at one of the steps 1e-4, 1e-5
    or 1e-6 of the value (a slot that changes steeply, or a branch of the
    set-up within the largest step, needs the smaller ones). Bar per step
    as test_setup_jvp_against_differences, the rounding term 1e5 ulp."""
    import torch

    from waveformx_b200 import _lib, ops
    from test_gpu_polarizations import draw_batch

    p = draw_batch(np.random.default_rng(53), 128)
    dev = cuda
    f_min = torch.tensor([20.0], dtype=torch.float64, device=dev)

    def rows(q):
        t = ops.setup("IMRPhenomXHM", torch.as_tensor(q, device=dev), f_min, precision=_lib.FP64)
        assert int(t.status.abs().sum()) == 0
        return t.table.cpu().numpy()

    dtable = ops.xhm_dtable(torch.as_tensor(p, device=dev), f_min).cpu().numpy()
    base = rows(p)
    parts = np.concatenate([np.zeros(72, int), np.ones(24, int), 2 + np.arange(4 * 112) // 112])
    for j in range(8):
        tangent = dtable[:, :, j]
        scale = np.stack([np.abs(tangent[:, parts == g]).max(axis=1) for g in range(6)], axis=1)[:, parts]
        ok = np.zeros_like(tangent, dtype=bool)
        for rel in (1e-4, 1e-5, 1e-6):
            h = rel * np.maximum(1.0, np.abs(p[:, j]))

            def at(k):
                q = p.copy()
                q[:, j] += k * h
                return rows(q)

            fd = (8.0 * (at(1) - at(-1)) - (at(2) - at(-2))) / (12.0 * h[:, None])
            bar = 1e-6 * np.abs(fd) + 1e-9 * scale + 1e5 * 2.2e-16 * np.abs(base) / h[:, None]
            ok |= np.abs(tangent - fd) <= bar
        bad = np.argwhere(~ok)
        assert bad.size == 0, [(j, b, k, tangent[b, k]) for b, k in bad[:5]]


@pytest.mark.parametrize("with_tc, binaries", [(False, "golden"), (True, "golden"), (False, "q20")])
def test_gradient_against_differences(cuda, with_tc, binaries):
    """ops.xhm_vjp (forward mode through the FP64 evaluation along the
    set-up's tangents) against central differences of the FP64 waveform, for
    a linear loss L = sum Re(conj(a) h+ + conj(c) hx), every parameter and
    t_c (at t_c, or at zero without it), for five of the golden draws, or two
    of them with f_ref = 0 and the mass ratios either side of 20. Bar: 1e-5
    of each component (2e-7 of the largest); along f_ref = 0 the gradient is
    zero (a nonzero f_ref is another reference frequency)."""
    import torch

    from waveformx_b200 import _lib, ops

    data = golden("xhm_random")
    p = data["params"][:5].copy() if binaries == "golden" else np.concatenate([data["params"][:2],
                                                                            JVP_BINARIES[1:4]])
    grid = np.geomspace(20.0, 600.0, 257)
    dev = cuda
    f64 = torch.as_tensor(grid, device=dev)
    tc = np.array([0.0, 0.01, -0.02, 0.005, 0.03]) if with_tc else None
    rng = np.random.default_rng(11)
    a = rng.normal(size=(5, len(grid))) + 1j * rng.normal(size=(5, len(grid)))
    c = rng.normal(size=(5, len(grid))) + 1j * rng.normal(size=(5, len(grid)))

    def loss(params, t):
        pt = torch.as_tensor(params, device=dev)
        table = ops.setup("IMRPhenomXHM", pt, f64[:1], precision=_lib.FP64).table
        tt = None if t is None else torch.as_tensor(t, device=dev)
        hp, hc = ops.polarizations("IMRPhenomXHM", table, f64, None, tt)
        hp, hc = hp.cpu().numpy(), hc.cpu().numpy()
        return np.sum((np.conj(a) * hp).real + (np.conj(c) * hc).real, axis=1)

    grad = ops.xhm_vjp(torch.as_tensor(p, device=dev), f64[:1], f64, None,
                       None if tc is None else torch.as_tensor(tc, device=dev),
                       torch.as_tensor(a, device=dev), torch.as_tensor(c, device=dev)).cpu().numpy()
    # fourth-order central differences, steps of 1e-7 of each value (the
    # phase moves by ~1e-3 rad over one: truncation ~1e-12)
    fd = np.zeros((5, 9))
    tc0 = np.zeros(5) if tc is None else tc  # (t_c's column: the derivative at t_c, 0 without)
    for j in range(9):
        x = p[:, j] if j < 8 else tc0
        h = 1e-7 * np.maximum(1.0, np.abs(x))

        def at(k):
            if j < 8:
                q = p.copy()
                q[:, j] += k * h
                return loss(q, tc)
            return loss(p, tc0 + k * h)

        fd[:, j] = (8.0 * (at(1) - at(-1)) - (at(2) - at(-2))) / (12.0 * h)
    zero = p[:, 7] == 0.0
    assert np.all(grad[zero, 7] == 0.0)
    fd[zero, 7] = 0.0
    for j in range(9):
        scale = np.max(np.abs(fd[:, j]))
        err = np.abs(grad[:, j] - fd[:, j])
        assert np.all(err <= 1e-5 * np.abs(fd[:, j]) + 2e-7 * scale), (j, grad[:, j], fd[:, j])


def test_modes_api(cuda):
    """modes("IMRPhenomXHM", ...): the reference's call (its
    ``_api.py:180-187``): the modes on the two-sided grid, h_{l,-m} at the
    positive frequencies equal to the reference's, h_{l,m}(-f) = (-1)^l
    conj(h_{l,-m}(f)), and their sum with the harmonics the reference's
    polarizations."""
    import waveformx_b200 as wb

    data = golden("xhm_random")
    grid = data["frequencies"]
    n = len(grid)
    for b in (0, 5, 17):
        p = data["params"][b]
        fm = wb.modes("IMRPhenomXHM", grid, mass_1=p[0], mass_2=p[1], spin_1=(0, 0, p[2]), spin_2=(0, 0, p[3]),
                      luminosity_distance=p[4], inclination=p[5], phi_ref=p[6], f_ref=p[7])
        np.testing.assert_array_equal(fm.frequencies, np.concatenate([-grid[::-1], grid]))
        for k, (ell, emm) in enumerate(((2, 2), (2, 1), (3, 3), (3, 2), (4, 4))):
            ref = data["modes"][b, k]
            assert _peak_relative(fm[(ell, -emm)][n:], ref) < 1e-9
            assert np.all(fm[(ell, -emm)][:n] == 0)
            sign = -1.0 if ell % 2 else 1.0
            assert _peak_relative(fm[(ell, emm)][:n], (sign * np.conj(ref))[::-1]) < 1e-9
        hp, hc = fm.polarizations()
        assert _peak_relative(hp, data["hplus"][b]) < 1e-9
        assert _peak_relative(hc, data["hcross"][b]) < 1e-9


def test_choose_fd_modes(cuda):
    """choose_fd_modes: LAL's two-sided uniform grid, the band's modes those
    of modes() on the band, zero below f_min and above the cutoff."""
    import waveformx_b200 as wb

    kw = dict(mass_1=36.0, mass_2=29.0, spin_1=(0, 0, 0.3), spin_2=(0, 0, -0.1), luminosity_distance=500.0,
              inclination=0.7, phi_ref=1.2)
    delta_f, f_min = 0.25, 20.0
    fm = wb.choose_fd_modes("IMRPhenomXHM", delta_f, f_min, **kw)
    freqs = np.asarray(fm.frequencies)
    n_full = (len(freqs) + 1) // 2
    assert freqs[n_full - 1] == 0.0 and np.allclose(np.diff(freqs), delta_f)
    f_cut = 0.3 / (65.0 * 4.925490947641267e-06)
    i_start, i_stop = int(f_min / delta_f), int(f_cut / delta_f) + 1
    band = np.arange(i_start, i_stop) * delta_f
    direct = wb.modes("IMRPhenomXHM", band, f_ref=f_min, **kw)
    for mode in ((2, -2), (3, -3), (3, -2)):
        h = np.asarray(fm[mode])[n_full - 1:]
        assert _peak_relative(h[i_start:i_stop], np.asarray(direct[mode])[len(band):]) < 1e-12
        assert np.all(h[:i_start] == 0) and np.all(h[i_stop:] == 0)


def test_refusals_are_nan(cuda):
    """Where LAL refuses a binary the waveform is NaN, as the reference's
    pure function (mass ratio 2000; reference_mf with f_ref != 0), and the
    batch API reports it, with the other rows intact."""
    import torch

    import waveformx_b200 as wb
    from waveformx_b200 import _lib, ops

    grid = np.geomspace(20.0, 500.0, 64)
    f = torch.as_tensor(grid, device=cuda)
    good = [36.0, 29.0, 0.3, -0.1, 500.0, 0.7, 1.2, 20.0]
    for bad, rmf, bit in (([2000.0, 1.0, 0.0, 0.0, 400.0, 0.4, 0.0, 20.0], None, 1), (good, 0.01, 32)):
        p = torch.as_tensor([good, bad], dtype=torch.float64, device=cuda)
        if rmf is not None:
            p[0, 7] = 0.0
        for precision in (_lib.FP64, _lib.FP32):
            t = ops.setup("IMRPhenomXHM", p, f[:1], reference_mf=rmf, precision=precision)
            status = t.status.cpu().numpy()
            assert status[0] == 0 and status[1] & bit
            ff = f if precision == _lib.FP64 else f.float()
            hp, hc, modes = ops.xhm_modes(t.table, ff)
            assert np.all(np.isfinite(hp[0].cpu().numpy())) and np.all(np.isnan(hp[1].cpu().numpy()))
    cols = dict(mass_1=[36.0, 2000.0], mass_2=[29.0, 1.0], spin_1z=[0.3, 0.0], spin_2z=[-0.1, 0.0],
                luminosity_distance=[500.0, 400.0])
    res = wb.batch_polarizations("IMRPhenomXHM", grid, cols, output="numpy")
    assert list(res.ok) == [True, False] and 1 in res.errors
    assert np.all(np.asarray(res.hplus)[1] == 0) and np.all(np.isfinite(np.asarray(res.hplus)[0]))


@pytest.mark.parametrize("approximant, fixture", [("IMRPhenomXHM", "xhm_cases"), ("IMRPhenomXAS", "xas_cases"),
                                                  ("IMRPhenomD", "phenomd_cases"), ("TaylorF2", "taylorf2_cases")])
def test_keyword_polarizations(cuda, approximant, fixture):
    """polarizations(approximant, frequencies, **binary): the reference's
    single-binary call (its ``_api.py:156-170``) against its golden vectors;
    the model's checks raise."""
    import waveformx_b200 as wb

    data = golden(fixture)
    for b in (1, 2):
        p = data["params"][b]
        f = data["frequencies"][b]
        hp, hc = wb.polarizations(approximant, f, mass_1=p[0], mass_2=p[1], spin_1=(0, 0, p[2]), spin_2=(0, 0, p[3]),
                                  luminosity_distance=p[4], inclination=p[5], phi_ref=p[6], f_ref=p[7])
        assert hp.dtype == np.complex128
        assert _peak_relative(hp, data["hplus"][b]) < 1e-9
        assert _peak_relative(hc, data["hcross"][b]) < 1e-9
    with pytest.raises(wb.InvalidParameterError):  # (a non-precessing model)
        wb.polarizations(approximant, f, mass_1=30.0, mass_2=20.0, spin_1=(0.5, 0, 0))
    if approximant in ("IMRPhenomXAS", "IMRPhenomXHM"):
        with pytest.raises(wb.InvalidParameterError):  # (IMRPhenomX's mass-ratio limit)
            wb.polarizations(approximant, f, mass_1=2000.0, mass_2=1.0)
