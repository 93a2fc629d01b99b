"""Handles used from several host threads at once.

Each handle owns its device buffers and streams, so a caller may drive two
handles from two threads -- e.g. to overlap one system's host copies with
another's evaluation.  The library's shared state (the operator-plan cache)
is locked.  Checked here: two evaluations running concurrently, each with
host copies in and out, give exactly the results the same handles give one
at a time.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_two_handles_on_two_threads(prec):
    from minimal_b200 import FMM, drand48_bodies, plummer_bodies

    inputs = [drand48_bodies(60000, 5), plummer_bodies(40000, 6)]
    handles = [FMM(P=10, ncrit=64, theta=0.4, precision=prec) for _ in inputs]
    alone = []
    for f, xq in zip(handles, inputs):  # one at a time
        f.set_bodies(xq)
        f.evaluate()
        alone.append(f.bodies())
    together = [[None] * 3 for _ in handles]
    errors = []

    def run(k):
        try:
            for rep in range(3):  # set_bodies (host -> device), evaluate, bodies (device -> host)
                handles[k].set_bodies(inputs[k])
                handles[k].evaluate()
                together[k][rep] = handles[k].bodies()
        except Exception as e:  # surfaced in the main thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=(k,)) for k in range(len(handles))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for k in range(len(handles)):
        for rep in range(3):
            assert np.array_equal(together[k][rep], alone[k])
    for f in handles:
        f.close()
