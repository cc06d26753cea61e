"""Host-buffer entry points: the asynchronous two-deep unit gives exactly
what the synchronous one gives, across slot reuse and with separate output
buffers."""
import pytest
import torch

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu


def _host(case):
    return [torch.from_numpy(g.copy()).pin_memory() for g in case.grids()]


def _split(gs, nt):
    return gs[:3], gs[3:3 + nt], gs[3 + nt:9 + nt], gs[9 + nt]


@pytest.mark.parametrize("prec", [api.FP64, api.MIXED])
def test_async_host_units_equal_sync(prec):
    cases = [synth.make_case(32, 24, 64, (0.0, 15.0, 30.0), 0.1, seed=s) for s in (41, 42, 43)]
    nt = cases[0].ntheta
    ctx = api.Context(cases[0], precision=prec)
    refs = []
    for c in cases:
        h = _host(c)
        ctx.posterior_unit_host(*_split(h, nt), prec)
        refs.append(h)
    ins = [_host(c) for c in cases]
    outs = [[torch.empty_like(g).pin_memory() for g in ins[0]] for _ in range(4)]
    order = [0, 1, 2, 0]  # four calls in flight two at a time, slots reused
    for call, k in enumerate(order):
        ctx.posterior_unit_host_async(_split(ins[k], nt), _split(outs[call], nt), prec)
    ctx.host_wait()
    for call, k in enumerate(order):
        for a, b in zip(outs[call][:9 + nt], refs[k][:9 + nt]):
            assert torch.equal(a, b), (call, k)
    for a, c in zip(ins[0], cases[0].grids()):  # inputs untouched
        assert torch.equal(a, torch.from_numpy(c))
