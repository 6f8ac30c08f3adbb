"""CPU checks of the learned-proposal oracle and of the weight packing.

* oracle/learned.py's hand-written gradients equal central finite
  differences of its loss (float64, relative 1e-6);
* the flux divergence conserves the total height exactly in exact arithmetic
  (float64 sums to ~1e-15);
* the packed operand layout is a permutation of the weights.
"""

import numpy as np

from oracle import learned as L


def test_oracle_gradients_equal_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(1, 6, 7, 3))
    ws = [rng.normal(scale=0.4, size=(3, 3, 3, 5)), rng.normal(scale=0.4, size=(3, 3, 5, 4))]
    tgt = rng.normal(size=(1, 6, 7))
    loss, grads, _ = L.loss_and_grads(x, ws, tgt, 0.7, 0.01)
    eps = 1e-6
    for li, w in enumerate(ws):
        for idx in [(0, 0, 0, 0), (1, 2, 1, 3), (2, 1, 2, 1), (1, 1, 0, 2)]:
            wp = [v.copy() for v in ws]
            wm = [v.copy() for v in ws]
            wp[li][idx] += eps
            wm[li][idx] -= eps
            fd = (L.loss_and_grads(x, wp, tgt, 0.7, 0.01)[0]
                  - L.loss_and_grads(x, wm, tgt, 0.7, 0.01)[0]) / (2 * eps)
            assert abs(fd - grads[li][idx]) <= 1e-6 * max(1.0, abs(fd)), (li, idx)


def test_divergence_conserves():
    rng = np.random.default_rng(1)
    f = rng.normal(size=(2, 9, 11, 4))
    assert abs(L.divergence(f, 0.3).sum()) < 1e-12


def test_pack_index_is_a_permutation():
    from soilb200 import learned
    for cin, cout in ((16, 32), (32, 32), (32, 16), (16, 16)):
        idx = learned.pack_index(cin, cout)
        assert idx.size == 9 * cin * cout
        assert np.array_equal(np.sort(idx), np.arange(9 * cin * cout))
