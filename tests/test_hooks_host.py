"""The device-side hook objects (pyclaw_b200.hooks) used as ordinary host
callbacks give exactly what the shock-bubble app's own callbacks give
(apps/euler_2d/shockbubble.py:68-124); no GPU needed."""
import numpy as np

import kat_setups as K
import pyclaw_b200 as pc


def _state(mx=12, my=8):
    x = pc.Dimension('x', 0.0, 2.0, mx)
    y = pc.Dimension('y', 0.0, 0.5, my)
    domain = pc.Domain([x, y])
    state = pc.State(domain, 5, 1)
    state.problem_data['gamma'] = K.GAMMA
    state.problem_data['gamma1'] = K.GAMMA1
    return domain, state


def test_fixed_state_bc_matches_the_app_callback():
    p, q, aux, run, bcs, src = K.shockbubble_setup(mx=12, my=8)
    rinf, vinf, einf = K._shock_state()
    domain, state = _state()
    rng = np.random.default_rng(0)
    qbc = rng.random((5, 16, 12))
    want = qbc.copy()
    bcs[(0, "lower")](want, 0.0)
    pc.hooks.FixedStateBC([rinf, rinf * vinf, 0., einf, 0.], side="lower")(state, domain.patch.dimensions[0], 0.0,
                                                                             qbc, 2)
    assert np.array_equal(qbc, want)
    up = rng.random((5, 16, 12))
    pc.hooks.FixedStateBC(np.arange(5.0), side="upper")(state, domain.patch.dimensions[1], 0.0, up, 2)
    assert np.array_equal(up[:, :, -2:], np.broadcast_to(np.arange(5.0)[:, None, None], (5, 16, 2)))


def test_radial_source_matches_the_app_callback():
    p, q, aux, run, bcs, src = K.shockbubble_setup(mx=12, my=8)
    domain, state = _state()
    state.q[...] = q
    state.aux[...] = aux
    want = np.array(q, order="F")
    src(want, 0.0037)
    pc.hooks.EulerRadialSource(radius_aux=0)(None, state, 0.0037)
    assert np.array_equal(state.q, want)
