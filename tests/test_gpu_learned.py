"""The learned coarse proposal in the pair path (ofc_set_coarse_net) with the trained weights shipped in the package.

* Where the proposal starts the fine stage inside its capture range, the refined field equals the plain POC path's
  (the refinement is the same; only its start differs): on held-out pairs of the training distribution the learned
  path's error against the known field (RMS) stays within 2e-3 px of the POC path's, and its valid share within 2 %.
  Both errors are the refinement's own (about 0.03-0.05 px on these fields, whose strains reach 15 %).
* What the network gains over the method without it (its speed is measured by bench.py and optflow_b200.measure):
  it keeps working where the displacement leaves POC's capture range (a 28 px translation with max_disp = 8, where
  POC's single 64 px window cannot reach): there the learned path's error is far smaller.
* The fallback: with a network that proposes 60 px everywhere, every tile fails its check, POC takes over and the
  result equals the plain path's bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rms(r, field, n):
    tu, tv = field.displacement(n, n)
    m = np.isfinite(r.ux)
    du, dv = r.ux[m] - tu[m], r.uy[m] - tv[m]
    return float(np.sqrt(np.mean(du * du + dv * dv))), float(m.mean())


@pytest.fixture(scope="module")
def engines():
    from optflow_b200 import Engine
    plain, learned = Engine(0), Engine(0)
    learned.set_coarse_net("default")
    yield plain, learned
    plain.close()
    learned.close()


def test_learned_path_matches_the_plain_path_on_held_out_pairs(engines):
    from optflow_b200 import Config, net, track_pair
    plain, learned = engines
    rng = np.random.default_rng(777)
    n = 512
    for _ in range(4):
        a, b, field = net.training_pair(rng, n, n, engine=plain)
        e0, v0 = _rms(track_pair(a, b, Config(), engine=plain), field, n)
        e1, v1 = _rms(track_pair(a, b, Config(), engine=learned), field, n)
        assert abs(e1 - e0) < 2e-3 and e1 < 0.2, (e0, e1)
        assert v1 > v0 - 0.02, (v0, v1)


def test_learned_path_reaches_beyond_pocs_capture_range(engines):
    from optflow_b200 import Config, synth, track_pair
    plain, learned = engines
    n = 512
    p = synth.make_pattern(n, n, seed=5, rmin=1.5, rmax=2.5)
    field = synth.Field(t=(28.0, -6.0), c=(n / 2, n / 2), A=((1.004, 0.0), (0.0, 0.998)))
    a = synth.degrade(synth.render(p, n, n, None, engine=plain), seed=1, noise=0.008, bits=8)
    b = synth.degrade(synth.render(p, n, n, field, engine=plain), seed=2, noise=0.008, bits=8)
    cfg = Config(max_disp=8.0)
    e0, v0 = _rms(track_pair(a, b, cfg, engine=plain), field, n)
    e1, v1 = _rms(track_pair(a, b, cfg, engine=learned), field, n)
    assert v1 > 0.5 and e1 < 0.05, (e1, v1)
    assert v1 > v0 or e1 < 0.2 * e0, (e0, v0, e1, v1)


def test_a_wrong_proposal_falls_back_to_poc_everywhere():
    from optflow_b200 import Config, Engine, net, track_pair
    rng = np.random.default_rng(4)
    a, b, _ = net.training_pair(rng, 256, 256)
    plain = Engine(0)
    wrong_eng = Engine(0)
    wrong = np.zeros(net.param_count(), np.float32)
    wrong[-16:-14] = 60.0  # the last layer's biases: the decoder proposes (60, 60) px at every cell
    wrong_eng.set_coarse_net(wrong, tile=64, max_low_share=0.0)
    r0 = track_pair(a, b, Config(), engine=plain)
    r1 = track_pair(a, b, Config(), engine=wrong_eng)
    st = wrong_eng.coarse_net_stats()
    assert st["pairs"] == 1 and st["fallback_pairs"] == 1 and st["failed_tiles"] == st["tiles"], st
    for k in ("ux", "uy", "conf"):
        np.testing.assert_array_equal(getattr(r1, k), getattr(r0, k))
    plain.close()
    wrong_eng.close()
