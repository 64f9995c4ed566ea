"""BSDF parity: the renderer's device BSDF code (ks_bsdf_eval / ks_bsdf_sample, compiled in the
fast-math shading unit) against the oracle's restatement of principled_bsdf.cpp, microfacet.h and
bsdf.cpp, per function, over every BSDF kind the library renders:

  * PrincipledBSDF with GGX and Beckmann, including the transmission lobes (specular_trans,
    diffuse_trans with forward scattering), index of refraction 1, 1.5 and 4, and outgoing
    directions below the surface (refraction from inside, the std::beta G2 of microfacet.h:79-89);
  * PrincipledBRDF with GGX and Beckmann (principled_bsdf.cpp:11-225);
  * Lambertian (bsdf.cpp:13-41).

Stated bounds (device against oracle, same inputs): eval f cos and pdf within a relative 2e-3 of
the larger value plus 1e-6 for 99.5 % of the (wo, wi) pairs and within 5e-2 for 99.95 %; samples:
the same decision (no sample / a sample) for 99.5 %, and where both sample, wi within 2e-3 and
weight and pdf within a relative 2e-3 for 99 %.  The shading unit's approximate division, square
root, exp/log/pow and the host libm's correctly rounded ones differ in the last bits; the loose
0.05 % tail is where such bits decide a lobe (a Fresnel term at total internal reflection, a cosine
at the horizon).  Exclusions: the unit flushes denormal intermediates to zero, so where the
oracle's f cos is below 1e-20 (grazing refraction) the device may return exactly 0 and, as
eval_and_pdf does for a zero value (principled_bsdf.cpp:297-307), pdf 0.  Glass at ior 1 is
degenerate in the reference: its reflection lobe is rounding noise (a Fresnel term of 0 evaluated
to 1e-16, absorbed by the absolute 1e-6), and the dielectric lobe's selection weight is the
Fresnel reflectance at wo (lobe_sample_weights, principled_bsdf.cpp:518-541), zero up to rounding,
so whether its pdf and samples exist at all is decided by rounding noise: there only f cos and the
sampled directions are compared.

The CPU half checks the oracle on its own: every sample's pdf equals eval_and_pdf's pdf of the
same direction, its weight equals f cos / pdf, and the mean weight matches f cos integrated
over the sphere by uniform sampling (the sampling routines draw from the density they report).
"""
import numpy as np
import pytest


def material(**kw):
    import keepsake_b200 as ks
    m = ks.MaterialDesc()
    m.basecolor[:] = kw.pop("basecolor", (0.7, 0.5, 0.3))
    m.roughness = kw.pop("roughness", 0.5)
    m.metallic = kw.pop("metallic", 0.0)
    m.ior = kw.pop("ior", 1.5)
    m.specular_r0_mul = kw.pop("specular_r0_mul", 0.5)
    m.specular_trans = kw.pop("specular_trans", 0.0)
    m.diffuse_trans = kw.pop("diffuse_trans", 0.0)
    m.diffuse_trans_fwd = kw.pop("diffuse_trans_fwd", 0.5)
    m.microfacet = kw.pop("microfacet", 0)
    m.bsdf = kw.pop("bsdf", 0)
    m.specular = kw.pop("specular", 0.5)
    assert not kw, kw
    return m


# name -> material fields
MATERIALS = {
    "diffuse": dict(roughness=1.0),
    "metal_ggx": dict(metallic=1.0, roughness=0.3),
    "metal_mixed": dict(metallic=0.4, roughness=0.6),
    "glass_ggx_ior15": dict(specular_trans=1.0, roughness=0.2, ior=1.5),
    "glass_ggx_ior1": dict(specular_trans=1.0, roughness=0.4, ior=1.0),
    "glass_ggx_ior4": dict(specular_trans=1.0, roughness=0.3, ior=4.0),
    "glass_half": dict(specular_trans=0.5, roughness=0.5, ior=1.5),
    "diffuse_trans_full": dict(diffuse_trans=1.0, diffuse_trans_fwd=0.0),
    "diffuse_trans_fwd": dict(diffuse_trans=0.5, diffuse_trans_fwd=0.7),
    "beckmann_plastic": dict(microfacet=1, roughness=0.4),
    "beckmann_metal": dict(microfacet=1, metallic=1.0, roughness=0.25),
    "beckmann_glass": dict(microfacet=1, specular_trans=1.0, roughness=0.3, ior=1.5),
    "brdf_ggx": dict(bsdf=1, roughness=0.35, metallic=0.3, specular=0.6),
    "brdf_beckmann": dict(bsdf=1, microfacet=1, roughness=0.5, metallic=0.0, specular=0.5),
    "brdf_metal": dict(bsdf=1, roughness=0.2, metallic=1.0),
    "lambertian": dict(bsdf=2, basecolor=(0.9, 0.6, 0.2)),
}


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def directions(n, seed, below=True):
    """Unit vectors over the whole sphere (below = True) or the upper hemisphere, with a share
    near the horizon and at the pole."""
    rng = np.random.default_rng(seed)
    d = unit(rng.normal(size=(n, 3)))
    if not below:
        d[:, 2] = np.abs(d[:, 2])
    d[: n // 50, 2] *= 1e-3  # grazing
    d[n // 50: n // 25] = [0.0, 0.0, 1.0]  # normal incidence
    return unit(d).astype(np.float32)


def close(a, b, rtol, atol=1e-30):
    """Per row: |a - b| <= rtol * max(|a|, |b|) + atol (largest component)."""
    a = np.atleast_2d(np.asarray(a, np.float64).T).T
    b = np.atleast_2d(np.asarray(b, np.float64).T).T
    scale = np.maximum(np.abs(a).max(-1), np.abs(b).max(-1))
    return np.abs(a - b).max(-1) <= rtol * scale + atol


# ---------------------------------------------------------------------------------------------
# oracle on its own (CPU)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", list(MATERIALS))
def test_oracle_sample_matches_eval_and_pdf(oracle, name):
    """Where eval_and_pdf sees the sampled direction (f cos > 0), its pdf is the pdf the sampler
    reported (to 1e-3: a peaked D recomputed from wo and wi loses a few bits) and the sample's
    weight is f cos / pdf.  Two properties of the reference are kept, not fixed: a forward-
    scattering diffuse-transmission lobe (diffuse_trans_fwd > 0.05) draws Henyey-Greenstein
    directions around -wo that can land on wo's side, where the sampler still counts that lobe's
    pdf and eval_and_pdf does not (principled_bsdf.cpp:349-356 against :395-421); and rough
    refraction at ior 1 (skipped here) sends wi to -wo up to rounding, where the generalised half
    vector wo + eta wi is rounding noise (exactly zero it is 0 / 0, which the reference asserts
    against, principled_bsdf.cpp:500; the library counts no transmission there)."""
    if name == "glass_ggx_ior1":
        pytest.skip("rough refraction at ior 1 is degenerate in the reference")
    m = material(**MATERIALS[name])
    n = 4000
    wo = directions(n, 1)
    u = np.random.default_rng(2).random((n, 3), dtype=np.float32)
    wi, w, pdf = oracle.bsdf_sample(m, wo, u)
    ok = pdf > 0
    assert ok.mean() > 0.2
    assert np.isfinite(w[ok]).all() and (w[ok] >= 0).all()
    if m.diffuse_trans > 0 and m.diffuse_trans_fwd > 0.05:
        ok &= wo[:, 2] * wi[:, 2] < 0
    f, p = oracle.bsdf_eval(m, wo[ok], wi[ok])
    seen = (f > 0).any(-1)
    assert seen.mean() > 0.99, (name, seen.mean())
    good = close(p[seen], pdf[ok][seen], 1e-3)
    assert good.mean() > 0.999, (name, good.mean())
    good = close(f[seen] / p[seen, None], w[ok][seen], 1e-3)
    assert good.mean() > 0.999, (name, good.mean())


def sampled_and_integrated(oracle, m, wo, rng, n=200_000):
    """(E[weight] of the sampler, f cos integrated over the sphere by uniform sampling, the
    combined standard error) for one outgoing direction."""
    wo = unit(np.asarray(wo, np.float64)).astype(np.float32)
    u = rng.random((n, 3), dtype=np.float32)
    _, w, _ = oracle.bsdf_sample(m, np.repeat(wo[None], n, 0), u)
    d = unit(rng.normal(size=(n, 3))).astype(np.float32)
    f, _ = oracle.bsdf_eval(m, np.repeat(wo[None], n, 0), d)
    se = f.std(0) * 4 * np.pi / np.sqrt(n) + w.std(0) / np.sqrt(n)
    return w.mean(0), f.mean(0) * 4 * np.pi, se


@pytest.mark.parametrize("name", ["diffuse", "metal_mixed", "glass_half", "diffuse_trans_full", "beckmann_plastic",
                                  "brdf_ggx", "brdf_beckmann", "lambertian"])
def test_oracle_sampling_density_integrates(oracle, name):
    """E[weight] over the sampler equals the integral of f cos over the sphere (uniform-sphere
    estimate), per wo: the sampler draws from the density it reports."""
    m = material(**MATERIALS[name])
    rng = np.random.default_rng(3)
    for wo in ([0.3, 0.2, 0.93], [0.8, -0.1, 0.3]):
        est_sample, est_uniform, se = sampled_and_integrated(oracle, m, wo, rng)
        assert (np.abs(est_sample - est_uniform) <= 5 * se + 2e-3).all(), (name, wo, est_sample, est_uniform)


def test_oracle_forward_diffuse_transmission_overcounts(oracle):
    """The reference's forward-scattering diffuse transmission (diffuse_trans_fwd > 0.05) draws
    Henyey-Greenstein directions around -wo, some on wo's side, and weighs them with the lobe's pdf
    that eval_and_pdf leaves out there (principled_bsdf.cpp:349-356 against :395-421): its sampled
    weights average above the integral of f cos.  The oracle and the library keep that estimator."""
    m = material(**MATERIALS["diffuse_trans_fwd"])
    est_sample, est_uniform, se = sampled_and_integrated(oracle, m, [0.3, 0.2, 0.93], np.random.default_rng(4))
    assert (est_sample > est_uniform + 10 * se).all(), (est_sample, est_uniform)


# ---------------------------------------------------------------------------------------------
# device BSDF code against the oracle (GPU)
# ---------------------------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", list(MATERIALS))
def test_bsdf_eval_matches_oracle(ctx, oracle, name):
    m = material(**MATERIALS[name])
    n = 20000
    wo = directions(n, 10)
    wi = directions(n, 11)
    f, p = ctx.bsdf_eval(m, wo, wi)
    of, op = oracle.bsdf_eval(m, wo, wi)
    assert np.isfinite(f).all() and np.isfinite(p).all()
    assert ((f > 0).any(-1) | (p >= 0)).all()
    # the fast-math shading unit flushes denormal results to zero: rows whose oracle value is
    # nonzero but below 1e-20 and whose device value is exactly zero (exact zeros, e.g. wi below an
    # opaque surface, are compared like every other row)
    tiny = np.abs(of).max(-1)
    flushed = (tiny > 0) & (tiny < 1e-20) & ~f.any(-1)
    assert flushed.mean() < 0.05
    keep = ~flushed
    checks = [(f, of, "f cos")]
    if m.ior != 1.0 or m.specular_trans == 0.0:
        checks.append((p[keep], op[keep], "pdf"))
    for got, want, what in checks:
        tight = close(got, want, 2e-3, 1e-6)
        loose = close(got, want, 5e-2, 1e-6)
        assert tight.mean() >= 0.995 and loose.mean() >= 0.9995, (name, what, tight.mean(), loose.mean())
    # both sides of the surface and both kinds of pairs are exercised
    assert (wo[:, 2] < 0).any() and ((wo[:, 2] * wi[:, 2]) < 0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(MATERIALS))
def test_bsdf_sample_matches_oracle(ctx, oracle, name):
    m = material(**MATERIALS[name])
    n = 20000
    wo = directions(n, 20)
    u = np.random.default_rng(21).random((n, 3), dtype=np.float32)
    wi, w, p = ctx.bsdf_sample(m, wo, u)
    owi, ow, op = oracle.bsdf_sample(m, wo, u)
    assert np.isfinite(wi).all() and np.isfinite(w).all()
    if m.ior != 1.0:
        assert np.isfinite(p).all()
    same = (p > 0) == (op > 0)
    degenerate = m.ior == 1.0 and m.specular_trans > 0.0
    assert degenerate or same.mean() >= 0.995, (name, same.mean())
    both = (p > 0) & (op > 0)
    assert both.sum() > (0.02 if degenerate else 0.2) * n
    dir_ok = np.abs(wi[both] - owi[both]).max(-1) <= 2e-3
    w_ok = close(w[both], ow[both], 2e-3)
    p_ok = close(p[both], op[both], 2e-3)
    checks = [(dir_ok, "wi")]
    if m.ior != 1.0:  # at ior 1 refraction sends wi to -wo: pdf and weight are rounding noise there
        checks += [(p_ok, "pdf"), (w_ok, "weight")]
    for ok, what in checks:
        assert ok.mean() >= 0.99, (name, what, ok.mean())


@pytest.mark.gpu
def test_bsdf_hooks_reject_bad_materials(ctx):
    import keepsake_b200 as ks
    wo = directions(4, 0)
    for bad in (dict(bsdf=3), dict(microfacet=2), dict(roughness=float("nan"))):
        with pytest.raises(ks.KsError) as e:
            ctx.bsdf_eval(material(**bad), wo, wo)
        assert e.value.status == 1
    f, p = ctx.bsdf_eval(material(), wo[:0], wo[:0])
    assert f.shape == (0, 3) and p.shape == (0,)
