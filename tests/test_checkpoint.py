"""Checkpoint / resume on the host: the fit state (vertices, Adam moments, step,
Faces_coeff, sigma) and the learned initialiser (network, optimiser, scheduler)
survive a torch.save / torch.load round trip bit for bit, and a resumed optimiser
takes the same next step as an uninterrupted one."""
import math
import types

import pytest
import torch

from deltamic_b200.fit import fit_state_dict, load_fit_state, load_fit_state_dict, save_fit_state
from deltamic_b200.learned import LearnedInit, load_checkpoint, save_checkpoint


def _fake_step(nv, seed, optimizer="adam"):
    g = torch.Generator().manual_seed(seed)
    v2 = (torch.rand(nv, 3, generator=g) if optimizer == "adam"
          else torch.rand(nv, generator=g))
    return types.SimpleNamespace(
        V=torch.randn(nv, 3, generator=g), m=torch.randn(nv, 3, generator=g), v=v2,
        t=torch.tensor([17], dtype=torch.int64), lr=2e-3, betas=(0.9, 0.99), eps=1e-8,
        optimizer=optimizer, graph=None)


@pytest.mark.parametrize("opt", ["adam", "vector_adam"])
def test_fit_state_round_trip(tmp_path, opt):
    a = _fake_step(50, 1, opt)
    c = torch.rand(96)
    sig = torch.diag(torch.tensor([1e-3, 1e-3, 4e-3]))
    p = tmp_path / "fit.pt"
    save_fit_state(p, a, faces_coeff=c, sigma=sig, iteration=17, loss=0.25)
    b = _fake_step(50, 2, opt)
    b.lr = 1.0
    st = load_fit_state(p, b)
    for k in ("V", "m", "v", "t"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    assert b.lr == a.lr and tuple(b.betas) == tuple(a.betas)
    assert torch.equal(st["faces_coeff"], c) and torch.equal(st["sigma"], sig)
    assert st["extra"] == {"iteration": 17, "loss": 0.25}
    with pytest.raises(ValueError, match="shape"):
        load_fit_state_dict(b, fit_state_dict(_fake_step(49, 3, opt)))
    other = fit_state_dict(_fake_step(50, 3, "vector_adam" if opt == "adam" else "adam"))
    with pytest.raises(ValueError, match="optimizer"):
        load_fit_state_dict(b, other)
    # a captured step keeps its optimiser settings: a state with others is refused
    b.graph = object()
    s2 = fit_state_dict(a)
    s2["lr"] = 5e-2
    with pytest.raises(ValueError, match="captured"):
        load_fit_state_dict(b, s2)


def test_learned_checkpoint_round_trip_and_resume(tmp_path):
    torch.manual_seed(0)
    m = LearnedInit(n_verts=42, hidden=32, seed=3)
    opt = torch.optim.Adam(m.parameters(), lr=1e-3)
    sched = torch.optim.lr_scheduler.LambdaLR(opt, lambda it: 0.5 * (1 + math.cos(it / 10)))

    def fake_step(model, o, s, k):
        g = torch.Generator().manual_seed(k)
        for q in model.parameters():
            q.grad = torch.randn(q.shape, generator=g)
        o.step()
        s.step()

    for k in range(3):
        fake_step(m, opt, sched, k)
    p = tmp_path / "net.pt"
    save_checkpoint(p, m, opt, sched, epoch=3)
    m2 = LearnedInit(n_verts=42, hidden=32, seed=9)
    opt2 = torch.optim.Adam(m2.parameters(), lr=1e-3)
    sched2 = torch.optim.lr_scheduler.LambdaLR(opt2, lambda it: 0.5 * (1 + math.cos(it / 10)))
    m2, extra = load_checkpoint(p, m2, opt2, sched2)
    assert extra == {"epoch": 3}
    for a, b in zip(m.state_dict().values(), m2.state_dict().values()):
        assert torch.equal(a, b)
    fake_step(m, opt, sched, 99)
    fake_step(m2, opt2, sched2, 99)
    for a, b in zip(m.parameters(), m2.parameters()):
        assert torch.equal(a, b)
    m3, _ = load_checkpoint(p)  # a fresh model of the saved size
    assert m3.n_verts == 42 and m3.fc1.out_features == 32
