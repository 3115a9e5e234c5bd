"""Known answers for the oracle's restatement of exTracer/ImTracer (si3d_procedures.f90:4090-4487)
with conservative tracers (ecomod = 0).  The reference ships no tracer test data, so the
restatement is pinned by properties its flux form guarantees in a closed basin:
  * mass: sum over wet cells of h * tracer at the start of a step equals the same sum one step
    later (the horizontal fluxes cancel between neighbours, the vertical ones between layers, and
    ImTracer's top-layer thickness is the one continuity implies);
  * free-stream preservation: a uniform tracer stays uniform (its fluxes are velocity x constant,
    whose divergence continuity balances, and vertical diffusion of a constant is zero).
"""
import numpy as np
import pytest


def _wet(o, top="k1"):
    kmz = o.geti("kmz")[:o.lm]
    K = np.arange(1, o.km1 + 1)[:, None]
    lo = o.geti("k1z")[:o.lm][None, :] if top == "k1z" else 2
    return (K >= lo) & (K <= kmz[None, :])


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_tracer_mass_is_conserved(tracer_dirs, oracle_lib, name):
    o = oracle_lib.OracleRun(tracer_dirs[name])
    wet = _wet(o)

    def mass(t):
        return float((o.get(f"tracerpp{t}")[:, :o.lm] * o.get("hp")[:, :o.lm] * wet).sum())

    m0 = [mass(t) for t in (1, 2, 3)]
    o.run(30)
    m1 = [mass(t) for t in (1, 2, 3)]
    for a, b in zip(m0, m1):
        assert abs(b - a) <= 1e-12 * a, (m0, m1)


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_uniform_tracer_stays_uniform(tracer_dirs, oracle_lib, name):
    o = oracle_lib.OracleRun(tracer_dirs[name])
    o.run(30)
    tr = o.get("tracer3")[:, :o.lm]
    assert np.abs(tr[_wet(o, "k1z")] - 0.5).max() <= 1e-13


def test_tracers_move_and_stay_bounded(tracer_dirs, oracle_lib):
    """The step and the band actually change under the flow, and the superbee scheme keeps them
    within their initial range (no new extrema beyond round-off; negatives are clipped)."""
    o = oracle_lib.OracleRun(tracer_dirs["t1"])
    wet = _wet(o)
    a0 = [o.get(f"tracer{t}")[:, :o.lm][wet] for t in (1, 2)]
    o.run(30)
    for t, a in zip((1, 2), a0):
        b = o.get(f"tracer{t}")[:, :o.lm][wet]
        assert np.abs(b - a).max() > 1e-6
        assert b.min() >= 0.0 and b.max() <= a.max() + 1e-12


def test_save_copies_tracer_to_tracerpp(tracer_dirs, oracle_lib):
    o = oracle_lib.OracleRun(tracer_dirs["t0"])
    o.run(2)
    for t in (1, 2, 3):
        np.testing.assert_array_equal(o.get(f"tracer{t}"), o.get(f"tracerpp{t}"))
