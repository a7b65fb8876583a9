"""The serving loop's admission rules on the host: a request larger than
the HBM budget is refused at submit, queued requests report their state,
and a request cannot be released before it has finished."""
import pytest

import shygpu
from shygpu import cases


def test_oversize_request_is_refused(channel):
    fp = shygpu.footprint([channel])
    srv = shygpu.Server(fp - 1, max_active=2, quantum_steps=5)
    with pytest.raises(shygpu.ShyError) as e:
        srv.submit(channel, 10)
    assert e.value.code == 9 and "exceeds the server's budget" in str(e.value)
    srv.close()


def test_queued_request_state(channel):
    srv = shygpu.Server(shygpu.footprint([channel]) * 4, max_active=2, quantum_steps=5)
    a = srv.submit(channel, 10)
    b = srv.submit(channel, 20)
    assert b == a + 1
    st, n, ts, ta, td = srv.status(a)
    assert st == shygpu.Server.QUEUED and n == 0 and ts >= 0 and ta < 0 and td < 0
    with pytest.raises(shygpu.ShyError):
        lib = shygpu.lib()
        shygpu.check(lib.shygpu_serve_release(srv.h, a), "release")
    with pytest.raises(shygpu.ShyError):
        srv.result(a)
    srv.close()
