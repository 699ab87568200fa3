"""One evaluate() split into pieces of output steps (the path that spreads a long instance over
GPUs), run piece by piece on one GPU: operators and times equal the whole call's bit for bit, and
the states, scanned per piece from the exchanged piece products, agree to rounding."""
import numpy as np
import pytest

import fields as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pieces(inst, n_pieces, **kw):
    from spinsim_b200.shard import Piece, incoming_states, piece_ranges
    from spinsim_b200 import _lib
    _, n, _, _ = _lib.normalise_steps(inst.time_start, inst.time_end, inst.time_step_integration,
                                      inst.time_step_output)
    pieces = [Piece(inst, f, c, **kw) for f, c in piece_ranges(n, n_pieces)]
    products = [p.product.cpu().numpy() for p in pieces]  # the exchange
    for p, psi in zip(pieces, incoming_states(products, inst.state_init)):
        p.finish(psi)
    res = [p.results() for p in pieces]
    return (np.concatenate([r.time for r in res]), np.concatenate([r.time_evolution for r in res]),
            np.concatenate([r.state for r in res]), np.concatenate([r.spin for r in res]))


@pytest.mark.parametrize("n_pieces", [1, 3, 7])
def test_split_user_field_spin_one(cuda, n_pieces):
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch, Instance
    sweep = [F.TAU * 1e3, F.TAU * 4e3]
    inst = Instance(ss.SpinQuantumNumber.ONE, 0.0, 3e-3, 100e-9, 1e-6, ss.SpinQuantumNumber.ONE.plus_z, sweep)
    whole = Batch([inst], get_field=F.rabi_one)
    whole.run()
    w = whole.result(0)
    t, u, s, sp = _pieces(inst, n_pieces, get_field=F.rabi_one)
    assert np.array_equal(t, w.time)
    assert np.array_equal(u, w.time_evolution)
    assert np.abs(s - w.state).max() < 1e-12
    assert np.abs(sp - w.spin).max() < 1e-12
    ot, ou, os_, osp = O.evaluate(3, O.Field(3), sweep, 0.0, 3e-3, 100e-9, 1e-6, ss.SpinQuantumNumber.ONE.plus_z)
    assert np.array_equal(t, ot)
    assert np.abs(s - os_).max() < 1e-10


def test_split_tones_fp32_bulk(cuda):
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch, Instance
    p = F.tone_parameters(np.random.default_rng(31))
    tones = {a: np.array([(p[4 + 24 * a + 3 * k], p[5 + 24 * a + 3 * k], p[6 + 24 * a + 3 * k]) for k in range(8)])
             for a in range(3)}
    inst = Instance(ss.SpinQuantumNumber.HALF, 0.0, 2e-3, 10e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z,
                    field=ss.ToneField(tones, bias=list(p[:4])))
    for prec in (ss.Precision.FP64, ss.Precision.FP32_BULK):
        whole = Batch([inst], precision=prec)
        whole.run()
        w = whole.result(0)
        t, u, s, _ = _pieces(inst, 5, precision=prec)
        assert np.array_equal(t, w.time)
        if prec == ss.Precision.FP64:
            assert np.array_equal(u, w.time_evolution)
            assert np.abs(s - w.state).max() < 1e-11
        else:
            # a piece's intervals pair up differently in the warps, so the FP64 synthesis rounds
            # differently and an FP32 residual can round the other way: far inside the form's 1e-6
            assert np.abs(u - w.time_evolution).max() < 1e-9
            assert np.abs(s - w.state).max() < 1e-9


def test_piece_out_of_range_rejected(cuda):
    import spinsim_b200 as ss
    from spinsim_b200.batch import Batch, Instance
    inst = Instance(ss.SpinQuantumNumber.HALF, 0.0, 10e-6, 100e-9, 1e-6, ss.SpinQuantumNumber.HALF.plus_z,
                    field=ss.ToneField({2: [[1.0, 1.0, 0.0]]}), intervals=(5, 6))
    with pytest.raises(ValueError):
        Batch([inst])
