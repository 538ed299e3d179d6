"""The step's own FP64 ln/exp (atanh series + Cody-Waite/Taylor, the same
routines the CUDA kernels use) against the platform's correctly rounded
double log/exp, and the F32 results they give for the friction power
max(wh, 1e-5) ** f32(7/3) and the Horton exponential against a rounding of
the exact double result."""
import numpy as np

import engine as oracle_engine


def ulps(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.spacing(np.abs(b))


def test_ln_and_exp_are_within_two_ulp_of_double():
    lib = oracle_engine.library()
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.exp(rng.uniform(-40, 40, 4000)), [1.0, 2.0, 0.5, 1e-300, 1e300, 1.0000001]])
    ln = np.array([lib.ora_ln(float(x)) for x in xs])
    assert ulps(ln[xs != 1.0], np.log(xs[xs != 1.0])).max() <= 2.0
    assert lib.ora_ln(1.0) == 0.0
    ys = np.concatenate([rng.uniform(-700, 700, 4000), [0.0, 1.0, -1.0, 1e-10]])
    ex = np.array([lib.ora_exp(float(y)) for y in ys])
    assert ulps(ex, np.exp(ys)).max() <= 2.0


def test_friction_power_and_horton_exp_round_like_the_exact_value():
    lib = oracle_engine.library()
    rng = np.random.default_rng(1)
    y = float(np.float32(7.0 / 3.0))
    wh = np.concatenate([np.float32(1e-5) * np.ones(1), np.exp(rng.uniform(np.log(1e-5), np.log(50.0), 20000))])
    wh = wh.astype(np.float32)
    got = np.array([lib.ora_powf(float(x), y) for x in wh], np.float32)
    exact = np.power(wh.astype(np.float64), y).astype(np.float32)
    diff = ulps(got, exact)
    assert diff.max() <= 1.0 and (diff == 0).mean() > 0.999
    a = (-rng.uniform(0, 40, 20000)).astype(np.float32)
    got = np.array([lib.ora_expf(float(v)) for v in a], np.float32)
    exact = np.exp(a.astype(np.float64)).astype(np.float32)
    diff = ulps(got, exact)
    assert diff.max() <= 1.0 and (diff == 0).mean() > 0.999


def test_f64_build_of_the_step_follows_the_f32_step_on_a_benign_case():
    """The F64 build (liboracle_f64.so, the precision study's reference) runs
    the same step: on 600 s of rain on a gentle 32 x 32 grid (no flow yet,
    water only accumulates) both builds take the same steps and agree to F32
    rounding."""
    import numpy as np
    from engine import OracleEngine
    from nhflood.plain import PlainRun
    from nhflood.workloads import plain_uniform_256
    w = plain_uniform_256(n=32)
    w.duration = 600
    runs = [PlainRun(w, lambda a, p, q=q: OracleEngine(a, p, precision=q)) for q in ('f32', 'f64')]
    for r in runs:
        while not r.done:
            r.advance()
    assert runs[0].steps == runs[1].steps == 600
    h32, h64 = runs[0].engine.get('depth'), runs[1].engine.get('depth')
    assert h64.dtype == np.float64 and h64.max() > 0.008
    np.testing.assert_allclose(h32, h64, rtol=0, atol=1e-6)
