"""Two engine contexts on one device.  The ring kernels' dynamic shared-memory
opt-in is an attribute of the kernel function on the device, which both
contexts share: a context that needs less must not lower what the other one
relies on."""
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200 import _lib
from qlatanneal_b200.instances import sk_dense

pytestmark = pytest.mark.gpu


def _run(n, seed):
    h, J = sk_dense(n, seed)
    model = qa.DenseIsing(h, J)
    sched = qa.SQASchedule.from_vectors([4.0, 4.0, 4.0], [1.0, 0.5, 0.1])
    res = qa.SQAAnnealer(model, sched, 32, 1).run_reads(1, 1, reads=2, seed=3)
    return [r.best_energy for r in res], model


def test_two_contexts_share_the_kernel_opt_in(monkeypatch):
    e1 = _lib.Engine.get(0)
    e2 = _lib.Engine(0)
    a, m1 = _run(512, 1)  # n=512, P=32: the +-1 kernel with ~111 KB of shared memory
    monkeypatch.setitem(_lib.Engine._engines, 0, e2)
    _, m2 = _run(384, 2)  # the same kernel with ~75 KB, from the other context
    m2.release()
    monkeypatch.setitem(_lib.Engine._engines, 0, e1)
    b, m3 = _run(512, 1)  # the first context again
    assert a == b
    m1.release()
    m3.release()
    e2.close()
