"""Host-side logic of the serving loop that needs no GPU: the page-locked
result arena hands out first-fit regions, takes them back, and falls back to
a buffer of its own when nothing fits."""
import torch

from atum_b200 import serving


def _unpinned(monkeypatch):
    real = torch.empty

    def empty(*a, **k):
        k.pop("pin_memory", None)
        return real(*a, **k)

    monkeypatch.setattr(torch, "empty", empty)


def test_result_arena_first_fit_and_fallback(monkeypatch):
    _unpinned(monkeypatch)
    R = serving._ResultArena(nbytes=8 * 100)
    a, ta = R.get(30)
    b, tb = R.get(50)
    assert (ta, tb) == ((0, 30), (30, 80)) and a.numel() == 30 and b.numel() == 50
    # the two views do not overlap
    a.fill_(1.0)
    b.fill_(2.0)
    assert float(a.sum()) == 30.0 and float(b.sum()) == 100.0
    c, tc = R.get(30)
    assert tc is None and R.fallbacks == 1 and c.numel() == 30
    R.put(ta)
    d, td = R.get(25)
    assert td == (0, 25)
    e, te = R.get(20)
    assert te == (80, 100)
    f, tf = R.get(6)  # the 5-double gap and the full end do not fit
    assert tf is None and R.fallbacks == 2
    for t in (tb, td, te):
        R.put(t)
    R.put(None)
    assert R.used == []
    g, tg = R.get(100)
    assert tg == (0, 100)


def test_result_arena_larger_than_arena(monkeypatch):
    _unpinned(monkeypatch)
    R = serving._ResultArena(nbytes=8 * 10)
    v, t = R.get(11)
    assert t is None and v.numel() == 11 and R.buf is None
