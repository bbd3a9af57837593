"""Learned lambda placement end to end on the batched engine, at toy size:
pilot and dense runs of a few perturbations, features and targets, the
network trained on the tensor cores, schedules predicted and used."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_placement_pipeline(tmp_path):
    from q_b200 import lambda_placement as L
    base, perts = L.make_perturbations(str(tmp_path), 4, seed=3, steps=1000)
    data = L.training_data(perts, steps_eq=50, steps_prod=200)
    F, T = data["features"], data["targets"]
    assert F.shape == (4, 12) and T.shape == (4, 11) and np.all(np.isfinite(F)) and np.all(np.isfinite(T))
    assert np.allclose(T.sum(1), 0.0, atol=1e-9)                       # centred log-spacings
    assert np.all(data["sigma_dense"] > 0)
    model = L.fit(F, T, iters=500, lr=3e-3)
    assert model.loss[-1] < 0.2 * model.loss[0]                       # fits 4 samples
    u = L.place(F[0], model)
    assert len(u) == 12 and u[0] == 0.0 and u[-1] == 1.0 and np.all(np.diff(u) > 0)
    assert np.allclose(u, L.positions_from_logits(model.predict_logits(F[:1])[0]))
    assert np.allclose(L.place(F[0], None), np.linspace(0, 1, 12))    # fallback: uniform
    p = tmp_path / "model.npz"
    model.save(str(p))
    assert np.allclose(L.Placement.load(str(p)).predict_logits(F), model.predict_logits(F))
    # the predicted schedule drives a batched run
    runs = L.sample([(perts[0].inp, u)], replicas=2, steps_eq=20, steps_prod=100)
    assert len(runs[0].dG) == 2 and np.all(np.isfinite(runs[0].dG)) and runs[0].gpu_seconds > 0


def test_network_improves_on_the_pilot_spacing_for_structured_profiles():
    """On sigma(u) profiles with bumps the 5-window pilot under-resolves, the
    network trained on the tensor cores places windows closer to the
    optimal spacing than the pilot's own interpolation, and far closer than
    uniform spacing (held-out samples)."""
    from q_b200 import lambda_placement as L
    F, T = L.structured_profiles(2400, seed=7)
    # steps and weight decay chosen on a validation split (a short grid keeps the test brief)
    model = L.fit(F[:2000], T[:2000], grid_iters=(50, 100, 200), grid_decay=(0.0, 0.1))
    assert model.selection["validation_mse"] < model.selection["validation_mse_pilot"]
    learned = np.mean((model.predict_logits(F[2000:]) - T[2000:]) ** 2)
    pilot = np.mean((np.array([L.spacing_logits(L.pilot_spacing(f)) for f in F[2000:]]) - T[2000:]) ** 2)
    uniform = np.mean(T[2000:] ** 2)
    assert learned < 0.85 * pilot and learned < 0.2 * uniform
    # an untrained network returns the pilot spacing
    untrained = L.fit(F[:50], T[:50], iters=1, lr=0.0)
    assert np.allclose(untrained.predict(F[:3]), [L.pilot_spacing(f) for f in F[:3]], atol=1e-9)
