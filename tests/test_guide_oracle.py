"""CPU checks of the learned-guide oracle (oracle/oracle_guide.py): the analytic gradient against
finite differences, the mixture density's normalisation, and bfloat16 rounding."""
import numpy as np
import pytest

from oracle import oracle_guide as og

BOX = [-1.0, -1.0, -1.0, 1.0, 1.0, 1.0]


def _unit(v):
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def random_records(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1, 1, (n, 3))
    nrm = _unit(rng.normal(size=(n, 3)))
    wo = _unit(rng.normal(size=(n, 3)))
    wi = _unit(rng.normal(size=(n, 3)))
    w = rng.exponential(1.0, n)
    w[::7] = 0.0
    return np.concatenate([pos, nrm, wo, wi, w[:, None]], axis=1)


def test_bf16_rounding_known_answers():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -7, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    got = og.bf16(vals)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins; 1 + 3*2^-8 rounds up to 1 + 2^-6
    assert got[0] == 1.0
    assert got[1] == 1.0
    assert got[2] == 1.0 + 2 ** -6
    assert got[3] == 1.0 + 2 ** -7
    assert got[4] == -2.5
    assert np.isfinite(got[5])
    assert got[6] >= 0.0


def test_encoding_layout():
    f = og.encode([[0.0, 0.5, -1.0]], [[0, 1, 0]], [[1, 0, 0]], BOX)[0]
    assert f.shape == (64,)
    assert f[63] == 1.0 and np.all(f[60:63] == 0.0)
    # position u = (0.5, 0.75, 0): k = 0 terms are sin/cos(pi u)
    assert f[0] == pytest.approx(np.sin(np.pi * 0.5))
    assert f[3] == pytest.approx(np.cos(np.pi * 0.75))
    assert f[5] == pytest.approx(1.0)
    assert np.allclose(f[30:36], [0, 1, 0, 1, 0, 0])


def test_gradient_matches_finite_differences():
    params = og.init_params(3)
    rec = random_records(96, 4)
    loss, grad = og.loss_and_grad(params, rec, BOX, use_bf16=False)
    assert loss == pytest.approx(og.loss_only(params, rec, BOX), rel=1e-12)
    rng = np.random.default_rng(5)
    mask = og.trainable_mask().reshape(-1)
    idx = rng.choice(np.flatnonzero(mask), 48, replace=False)
    for p in idx:
        h = 1e-6
        a = params.copy()
        b = params.copy()
        a[p] += h
        b[p] -= h
        fd = (og.loss_only(a, rec, BOX) - og.loss_only(b, rec, BOX)) / (2 * h)
        assert grad[p] == pytest.approx(fd, rel=1e-4, abs=1e-8), p
    assert np.all(grad[~mask] == 0.0)


def test_mixture_pdf_integrates_to_one():
    rng = np.random.default_rng(6)
    raw = rng.normal(size=(1, 40))
    raw[0, 8:16] = rng.uniform(-2, 5, 8)
    # Fibonacci sphere quadrature
    m = 400000
    k = np.arange(m) + 0.5
    z = 1 - 2 * k / m
    phi = np.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    w = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    p = og.mixture_pdf(np.repeat(raw, m, axis=0), w)
    assert np.mean(p) * 4 * np.pi == pytest.approx(1.0, rel=2e-3)


def test_bf16_gradient_close_to_exact():
    params = og.init_params(7)
    rec = random_records(256, 8)
    _, g64 = og.loss_and_grad(params, rec, BOX, use_bf16=False)
    _, g16 = og.loss_and_grad(params, rec, BOX, use_bf16=True)
    rel = np.linalg.norm(g16 - g64) / np.linalg.norm(g64)
    assert rel < 0.05


def test_metal_density_matches_the_reference_sampler():
    """The density the learned guide's one-sample MIS uses at rough metallic vertices.  For random
    surface frames and rays, the reference's metallic bounce (restated in numpy, with to_onb as the
    reference writes it) is histogrammed over (cos, phi) bins of a frame centred on its
    mean direction, out to the widest sample, and each bin's count agrees with the derived density
    integrated over the bin; the density integrates to 1 over the hemisphere (uniform Monte Carlo)."""
    rng = np.random.default_rng(4)
    cases = []
    for k in range(4):
        n0 = rng.normal(size=3)
        n0 /= np.linalg.norm(n0)
        tg = np.cross(n0, rng.normal(size=3))
        tg /= np.linalg.norm(tg)
        rd = rng.normal(size=3)
        rd -= (2.0 * max(rd @ n0, 0.0) + 0.2) * n0  # the normal faces the ray
        rd /= np.linalg.norm(rd)
        cases.append((rd, n0, tg, [0.35, 0.3, 0.6, 0.15][k], [0.2, 0.3, 0.9, 0.5][k]))
    for rd, n0, tg, ax, ay in cases:
        V, R, _ = og.metal_frame(rd, n0, tg)
        u = rng.random((2, 2_000_000))
        ct, ph = u[0], 2.0 * np.pi * u[1]
        st = np.sqrt(1.0 - ct ** 2)
        uni = np.stack([st * np.cos(ph), ct, st * np.sin(ph)], 1)
        assert abs(og.metal_pdf(V, R, ax, ay, uni).mean() * 2.0 * np.pi - 1.0) < 0.03  # a few sigma of this estimate
        n = 1_000_000
        d = og.metal_sample(V, R, ax, ay, rng.random(n), rng.random(n))
        c = d.mean(0)
        c /= np.linalg.norm(c)
        e1 = np.cross(c, [1.0, 0.0, 0.0] if abs(c[0]) < 0.9 else [0.0, 1.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(c, e1)
        cmin = (d @ c).min() - 1e-6
        nt, npb, sub = 12, 24, 24
        H, te, pe = np.histogram2d(d @ c, np.arctan2(d @ e2, d @ e1), bins=[nt, npb], range=[[cmin, 1.0], [-np.pi, np.pi]])
        cs = (np.arange(sub) + 0.5) / sub
        exp = np.zeros_like(H)
        for i in range(nt):
            C = te[i] + cs * (te[i + 1] - te[i])
            for j in range(npb):
                P = pe[j] + cs * (pe[j + 1] - pe[j])
                CC, PP = np.meshgrid(C, P, indexing="ij")
                S = np.sqrt(np.clip(1.0 - CC ** 2, 0.0, 1.0))
                o = (CC[..., None] * c + S[..., None] * (np.cos(PP)[..., None] * e1 + np.sin(PP)[..., None] * e2)).reshape(-1, 3)
                exp[i, j] = og.metal_pdf(V, R, ax, ay, o).mean() * (te[i + 1] - te[i]) * (pe[j + 1] - pe[j]) * n
        assert abs(exp.sum() / n - 1.0) < 0.02, exp.sum() / n  # all of the density lies where the samples do
        m = exp > 400
        rel = np.abs(H[m] - exp[m]) / exp[m]
        assert H[m].sum() / n > 0.8 and np.median(rel) < 0.03, (H[m].sum() / n, np.median(rel))
