"""Checkpoint / resume of surrogate training (dosecuda_b200.surrogate.train).

A run interrupted mid-epoch and resumed from its training checkpoint (in a
fresh network object with other initial weights) must continue the
uninterrupted run: same weights, Adam moments and step counts at the
checkpoint, the same sample order afterwards, and final weights equal to the
straight run's up to the run-to-run effect of the weight-gradient kernels'
atomic (order-dependent) fp32 sums.  That effect is measured here by a second
straight run: Adam turns sign noise in near-zero gradient elements into
full-size steps, so two straight runs already differ visibly."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _flat(net):
    return torch.cat([v.detach().reshape(-1).double() for v in net.params.values()])


def test_resumed_training_continues_the_straight_run(tmp_path):
    from dosecuda_b200.surrogate import Dataset, SampleMaker, SurrogateNet, load_training_state, train
    maker = SampleMaker(shape=(64, 64, 64))
    data = Dataset(maker, range(6), dose_unit=2.0)
    kw = dict(epochs=3, lr=1e-3, seed=7, max_steps=14)
    p0 = _flat(SurrogateNet(seed=1))

    def logger(log):
        return lambda step, ep, i, lr: log.append((step, ep, i, lr))

    log_a, log_b, log_c = [], [], []
    straight = SurrogateNet(seed=1)
    train(straight, data, on_step=logger(log_a), **kw)
    again = SurrogateNet(seed=1)
    train(again, data, **kw)

    first = SurrogateNet(seed=1)
    path = tmp_path / "train_state.pt"
    train(first, data, state_path=str(path), session_steps=8, on_step=logger(log_b), **kw)
    blob = load_training_state(path)
    pr = blob["progress"]
    assert (pr["step"], pr["epoch"], pr["pos"]) == (8, 1, 2)
    for k, v in first.params.items():
        assert torch.equal(blob["trainer"]["params"][k], v.detach().cpu())
        assert float(blob["trainer"]["adam"][k]["step"]) == 8.0

    resumed = SurrogateNet(seed=99)  # everything must come from the checkpoint
    train(resumed, data, state_path=str(path), resume=str(path), on_step=logger(log_c), **kw)
    pr2 = load_training_state(path)["progress"]
    assert pr2["step"] == 14
    # same samples, epochs and learning rates, step for step
    assert len(log_a) == 14 and log_a == log_b + log_c

    other_order = SurrogateNet(seed=1)
    train(other_order, data, **dict(kw, seed=8))

    a = _flat(straight)
    move = (a - p0).norm().item()
    noise = (_flat(again) - a).norm().item()
    diff = (_flat(resumed) - a).norm().item()
    ctrl = (_flat(other_order) - a).norm().item()
    assert move > 0 and noise < 0.25 * move, (noise, move)
    assert diff < 2.0 * noise + 1e-3 * move, (diff, noise, move)
    assert diff < 0.5 * ctrl, (diff, ctrl)
